"""Builds the CPU test double of the C ABI (tests/fake_capi.c) into tests/_build/."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "fake_capi.c"
LIB = HERE / "_build" / "libfake_capi.so"


def build() -> str:
    deps = [SRC, HERE.parent / "oracle" / "replace_oracle.c"]
    if not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        LIB.parent.mkdir(parents=True, exist_ok=True)
        gcc = shutil.which("gcc") or "cc"
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run([gcc, "-O2", "-shared", "-fPIC", "-o", str(tmp), str(SRC)], check=True)
        tmp.replace(LIB)
    return str(LIB)
