"""Build libcuda_replace.so in-tree for sm_100a (B200).

The library is a plain C-ABI shared object (no Python or torch symbols), so the same
file is loaded by this package's ctypes wrapper and by the original
cuda_replace_wrapper.py. Usage: ``python -m cuda_replace_b200.build [--ptxas-v]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
LIB_NAME = "libcuda_replace.so"
LIB_PATH = PKG_DIR / LIB_NAME
SOURCES = ["replace_kernels.cu", "capi.cu", "noalloc.cu", "stream.cu", "batch.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libcuda_replace.so")
    return cand


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    deps = [CSRC / s for s in SOURCES] + [CSRC / "replace_kernels.h", CSRC / "host_pool.h", REPO_DIR / "include" / "cuda_replace.h"]
    if not force and not ptxas_verbose and not _stale(LIB_PATH, deps):
        return LIB_PATH
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [
        nvcc_path(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-fvisibility=hidden",
        *ARCH_FLAGS, "-lineinfo", "-I", str(REPO_DIR / "include"), "-I", str(CSRC),
        "-o", str(tmp), *[str(CSRC / s) for s in SOURCES],
    ]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    env = dict(os.environ)
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    path = build(force=True, ptxas_verbose="--ptxas-v" in sys.argv)
    print(path)
