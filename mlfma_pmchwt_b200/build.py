"""Builds the in-tree shared library ``libmlfma_pmchwt.so`` for sm_100a.

The library holds the whole product: host setup (C++), the CUDA kernels and
the C ABI declared in ``include/mlfma_pmchwt.h``. It is compiled with nvcc
directly (no JIT cache), so the ``.so`` sits next to this file and travels
with the source tree.

    python -m mlfma_pmchwt_b200.build          # incremental
    python -m mlfma_pmchwt_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libmlfma_pmchwt.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden,-ffp-contract=off",
    "-I", str(ROOT / "include"),
]


# Per-file flags. The near-field integrals take branches on near-zero
# geometric quantities against absolute thresholds (the singular-term
# extraction of Code/Operator.h); fused multiply-adds change those quantities
# in the last bits and can flip a branch, so that file is compiled with
# separately rounded multiplies and adds, like the reference's own build.
FILE_FLAGS = {"setup_kernels.cu": ["-fmad=false"]}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def host_cxx() -> str:
    # The container exports CXX as a wrapper without OpenMP specs; use the
    # system compiler for the host half of nvcc.
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "mlfma_pmchwt.h"])


def _compile(src: Path, force: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    newest_dep = max(p.stat().st_mtime for p in headers() + [src])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc(), "-ccbin", host_cxx(), *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[3:3] = ["-x", "cu"]
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), "-ccbin", host_cxx(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-cudart", "static"]
        subprocess.run(cmd, check=True)
    if verbose:
        print(f"built {LIB}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    build(force=args.force, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
