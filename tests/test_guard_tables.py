"""The guard tables of a post-collision BC list (csrc/guards.h, built on the host by boxes and
pools) against an independent restatement of their rule. For every list node Y and every cut
direction f (q in [0, 1]), the node X = Y + c_f (wrapped on periodic axes, dropped past a wall)
gets bit inv(f) in its mask when X is in the list: Y's write for f lands in the slot that X reads
as its post-collision population inv(f). first[] numbers the saved values in list order. Checked
on the porous blocks of the serving workload, whose sphere lists have such links, and on a list
with random q that reaches across the periodic and non-periodic faces."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from virtualfluids_b200.workloads import _CX, _CY, _CZ, porous_block_bcs

ROOT = Path(__file__).resolve().parent.parent
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
INV = np.array([0] + [d + 1 if d % 2 else d - 1 for d in range(1, 19)] + [45 - d for d in range(19, 27)])


@pytest.fixture(scope="module")
def guard_exe(tmp_path_factory):
    if not Path(NVCC).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path_factory.mktemp("guards") / "guard_tables_check"
    subprocess.run([NVCC, "-std=c++17", "--expt-relaxed-constexpr", f"-I{ROOT / 'virtualfluids_b200' / 'csrc'}",
                    str(ROOT / "tests" / "guard_tables_check.cu"), "-o", str(exe)], check=True, timeout=300)
    return exe


def _library_tables(exe, tmp_path, k, q, dims, periodic):
    src, dst = tmp_path / "list.bin", tmp_path / "table.bin"
    n = k.size
    bits = sum(1 << a for a in range(3) if periodic[a])
    with open(src, "wb") as f:
        f.write(np.array([n, *dims, bits], dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(k, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(q, dtype="<f8").tobytes())
    subprocess.run([str(exe), str(src), str(dst)], check=True, timeout=120)
    out = np.fromfile(dst, dtype="<u4")
    return int(out[0]), out[1:1 + n], out[1 + n:1 + 2 * n]


def _restated_tables(k, q, dims, periodic):
    nx, ny, nz = dims
    n = k.size
    pos = {int(v): i for i, v in enumerate(k)}
    x, y, z = k % nx, (k // nx) % ny, k // (nx * ny)
    mask = np.zeros(n, dtype=np.uint32)
    for f in range(1, 27):
        cut = (q[f] >= 0.0) & (q[f] <= 1.0)
        c = [x + _CX[f], y + _CY[f], z + _CZ[f]]
        ok = cut.copy()
        for a, e in enumerate(dims):
            out = (c[a] < 0) | (c[a] >= e)
            if not periodic[a]:
                ok &= ~out
            c[a] = c[a] % e
        kk = c[0] + nx * (c[1] + ny * c[2])
        for j in np.nonzero(ok)[0]:
            i = pos.get(int(kk[j]))
            if i is not None:
                mask[i] |= np.uint32(1 << int(INV[f]))
    counts = np.array([bin(int(m)).count("1") for m in mask], dtype=np.uint32)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    return int(counts.sum()), mask, first


@pytest.mark.parametrize("side,seed", [(24, 3), (32, 11)])
def test_guard_tables_of_porous_blocks(guard_exe, tmp_path, side, seed):
    g = porous_block_bcs(side, seed, porosity=0.75)
    k, q = g["bcs"]["noslip"]
    got = _library_tables(guard_exe, tmp_path, k, q, g["shape"], (False, True, True))
    want = _restated_tables(k, q, g["shape"], (False, True, True))
    assert got[0] == want[0] > 0
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])


@pytest.mark.parametrize("periodic", [(True, True, True), (False, True, False), (False, False, False)])
def test_guard_tables_of_random_lists_across_faces(guard_exe, tmp_path, periodic):
    rng = np.random.default_rng(7)
    dims = (9, 7, 6)
    n_all = dims[0] * dims[1] * dims[2]
    k = np.sort(rng.choice(n_all, size=n_all // 2, replace=False)).astype(np.int32)
    q = np.where(rng.random((27, k.size)) < 0.3, rng.random((27, k.size)), -1.0)
    q[0] = -1.0
    q[1, :3] = 0.0       # the ends of [0, 1] count as cut
    q[2, :3] = 1.0
    got = _library_tables(guard_exe, tmp_path, k, q, dims, periodic)
    want = _restated_tables(k, q, dims, periodic)
    assert got[0] == want[0] > 0
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
