"""Build recipe of the native library ``libvfb.so`` (CUDA kernels for sm_100a + the C ABI).

Every translation unit under ``csrc/`` is compiled by nvcc for ``sm_100a`` into the package
directory, so the shared object travels with the source tree. The ``k_exact_*`` units are
compiled without FMA contraction (``-fmad=false``): they are the bit-reproducible arithmetic
variant. ``build(checked=True)`` (``python -m virtualfluids_b200.build --checked``) makes
``libvfb_checked.so``, the same sources with ``-DVFB_BOUNDS_CHECK``: every node index taken from a
caller's array is checked against its level's node count (vfb_bounds_check_status). Run
``python -m virtualfluids_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libvfb.so"
BUILD_CHECKED = PKG / "_build_checked"
LIB_CHECKED = PKG / "libvfb_checked.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}"]


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _flags(src: Path, checked: bool = False):
    flags = list(COMMON) + ARCH
    if src.name.startswith("k_exact_"):
        flags.append("-fmad=false")
    if checked:
        flags.append("-DVFB_BOUNDS_CHECK")
    return flags


def _needs(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool, checked: bool = False):
    obj = (BUILD_CHECKED if checked else BUILD) / (src.stem + ".o")
    if not _needs(obj, src):
        return obj
    cmd = [NVCC] + _flags(src, checked) + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False, jobs: int | None = None, checked: bool = False) -> Path:
    """Compile and link ``libvfb.so`` (``libvfb_checked.so`` with checked=True); returns its path.
    Incremental on file times."""
    out_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    out_dir.mkdir(exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, checked), srcs))
    if not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(lib)] + [str(o) for o in objs] + ["-lcudart_static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, checked="--checked" in sys.argv))
