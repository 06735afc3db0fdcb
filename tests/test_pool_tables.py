"""The host tables of a pool domain (csrc/pool_tables.h) against a restatement of their contract
with the pool kernels, on the host:

* no-slip link tables: per node the mask of directions with q in [0, 1] in the pool's real type
  (q slightly above 1 in double can round to 1 in float and then counts), per 32 nodes the links
  of the nodes before them, and the link q in the order a warp of pool_noslip_kernel lists its
  links (direction by direction, lanes ascending), so that link l of chunk c reads q[first[c] + l];
* the collision's fluid-node queue: on for porous blocks, off for the ducts of the batch workload.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from virtualfluids_b200.workloads import porous_block_bcs

ROOT = Path(__file__).resolve().parent.parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    if not Path(NVCC).exists():
        pytest.skip("nvcc not available")
    path = tmp_path_factory.mktemp("pool_tables") / "pool_tables_check"
    subprocess.run([NVCC, "-std=c++17", "--expt-relaxed-constexpr", f"-I{ROOT / 'virtualfluids_b200' / 'csrc'}",
                    str(ROOT / "tests" / "pool_tables_check.cu"), "-o", str(path)], check=True, timeout=300)
    return path


def _links(exe, tmp_path, q, wide):
    n = q.shape[1]
    src, dst = tmp_path / "q.bin", tmp_path / "links.bin"
    with open(src, "wb") as f:
        f.write(np.array([n, int(wide)], dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(q, dtype="<f8").tobytes())
    subprocess.run([str(exe), "links", str(src), str(dst)], check=True, timeout=120)
    raw = dst.read_bytes()
    links = int(np.frombuffer(raw[:8], dtype="<u8")[0])
    m = n + (n + 31) // 32
    cut_first = np.frombuffer(raw[8:8 + 4 * m], dtype="<u4")
    link_q = np.frombuffer(raw[8 + 4 * m:], dtype="<f8" if wide else "<f4")
    return links, cut_first[:n], cut_first[n:], link_q


def _kernel_order(cut, n):
    """(node, direction) of every link, chunk by chunk as the kernel's warps list them."""
    out = []
    for c0 in range(0, n, 32):
        lanes = range(c0, min(n, c0 + 32))
        for d in range(1, 27):
            out += [(i, d) for i in lanes if (int(cut[i]) >> d) & 1]
    return out


@pytest.mark.parametrize("wide", [True, False], ids=["f64", "f32"])
def test_link_tables_follow_the_kernel_order(exe, tmp_path, wide):
    rng = np.random.default_rng(3)
    n = 100                                   # three full chunks and a ragged one
    q = np.where(rng.random((27, n)) < 0.25, rng.random((27, n)), -1.0)
    q[0] = 0.5                                # direction 0 is never a link
    q[3, :4] = [0.0, 1.0, 1.0 + 1e-12, -1e-12]
    links, cut, first, link_q = _links(exe, tmp_path, q, wide)
    qt = q if wide else q.astype(np.float32)
    active = (qt >= 0) & (qt <= 1)
    active[0] = False
    want_cut = (active.astype(np.uint64) << np.arange(27, dtype=np.uint64)[:, None]).sum(axis=0)
    assert np.array_equal(cut.astype(np.uint64), want_cut)
    assert links == int(active.sum()) == link_q.size
    per_node = active.sum(axis=0)
    assert np.array_equal(first, np.array([per_node[:c0].sum() for c0 in range(0, n, 32)]))
    # q[3] slightly above 1 rounds to 1 in float, so it is a link there and not in double
    assert bool((int(cut[2]) >> 3) & 1) == (not wide)
    order = _kernel_order(cut, n)
    for c, c0 in enumerate(range(0, n, 32)):
        chunk = [(i, d) for (i, d) in order if c0 <= i < c0 + 32]
        for l, (i, d) in enumerate(chunk):
            assert link_q[first[c] + l] == qt[d, i]


def _compact(exe, tmp_path, mask):
    src, dst = tmp_path / "mask.bin", tmp_path / "flag.bin"
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    with open(src, "wb") as f:
        f.write(np.array([m.size], dtype="<i8").tobytes())
        f.write(m.tobytes())
    subprocess.run([str(exe), "compact", str(src), str(dst)], check=True, timeout=120)
    return dst.read_bytes() == b"\x01"


def test_fluid_node_queue_for_porous_blocks_not_for_ducts(exe, tmp_path):
    assert _compact(exe, tmp_path, porous_block_bcs(32, 5, porosity=0.75)["mask"])
    for side in (16, 40, 96):
        nz = ny = side
        nx = side
        y = np.arange(ny)[None, :, None]
        z = np.arange(nz)[:, None, None]
        wall = (y == 0) | (y == ny - 1) | (z == 0) | (z == nz - 1)
        duct = np.broadcast_to(~wall, (nz, ny, nx))
        assert not _compact(exe, tmp_path, duct)
    assert not _compact(exe, tmp_path, np.zeros(64, dtype=np.uint8))
