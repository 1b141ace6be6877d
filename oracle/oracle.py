"""TEST INFRASTRUCTURE ONLY - the checker for libcuda_replace.so.

Ground truth is CPython's ``bytes.replace`` (chained once per pair for batches), which is
the check the reference itself uses (test/test.py:102-112 and 150-161). Beside it sits a
restatement of the reference's algorithm in C (``replace_oracle.c``: the seeded greedy of
cuda_replace.cu:938-968, the query of cuda_replace.cu:1825-1897), loaded here with ctypes,
and a pure-Python restatement for small cases. Only tests/, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of bench.py may use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path
from typing import Iterable, Sequence, Tuple

HERE = Path(__file__).resolve().parent
SRC = HERE / "replace_oracle.c"
LIB = HERE / "_build" / "libreplace_oracle.so"

_lib = None


def build_oracle(force: bool = False) -> Path:
    """Compile replace_oracle.c with gcc into oracle/_build/."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        raise RuntimeError("gcc is required to build the C oracle")
    LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([gcc, "-O2", "-shared", "-fPIC", "-o", str(tmp), str(SRC)], check=True)
    tmp.replace(LIB)
    return LIB


def _load():
    global _lib
    if _lib is None:
        path = LIB if LIB.exists() else build_oracle()
        lib = C.CDLL(str(path))
        i64, p8, pi64 = C.c_int64, C.c_char_p, C.POINTER(C.c_int64)
        lib.oracle_replace_len.argtypes = [p8, i64, p8, i64, i64, i64, pi64, pi64]
        lib.oracle_replace_len.restype = i64
        lib.oracle_replace.argtypes = [p8, i64, p8, i64, p8, i64, i64, C.c_void_p, i64, pi64, pi64]
        lib.oracle_replace.restype = i64
        lib.oracle_kept_positions.argtypes = [p8, i64, p8, i64, i64, pi64, i64]
        lib.oracle_kept_positions.restype = i64
        lib.oracle_query_prefix.argtypes = [p8, i64, p8, i64, i64, i64, pi64, pi64]
        lib.oracle_query_prefix.restype = None
        _lib = lib
    return _lib


def block_before_from_seed(prev_last_rel: int | None, L: int) -> int:
    """Seeded carry-in: candidates before prev_last_rel + L are blocked (cuda_replace.cu:938-968)."""
    if prev_last_rel is None or L == 0:
        return 0
    return max(0, prev_last_rel + L)


def replace(src: bytes, pat: bytes, rep: bytes, block_before: int = 0) -> Tuple[bytes, int, int]:
    """One replace with the C restatement. Returns (output, kept, last kept start or -1)."""
    lib = _load()
    kept, last = C.c_int64(0), C.c_int64(-1)
    n = lib.oracle_replace_len(src, len(src), pat, len(pat), len(rep), block_before, None, None)
    buf = C.create_string_buffer(max(n, 1))
    got = lib.oracle_replace(src, len(src), pat, len(pat), rep, len(rep), block_before,
                             C.cast(buf, C.c_void_p), n, C.byref(kept), C.byref(last))
    assert got == n, (got, n)
    return buf.raw[:n], kept.value, last.value


def replace_len(src: bytes, pat: bytes, rep_len: int, block_before: int = 0) -> Tuple[int, int, int]:
    lib = _load()
    kept, last = C.c_int64(0), C.c_int64(-1)
    n = lib.oracle_replace_len(src, len(src), pat, len(pat), rep_len, block_before,
                               C.byref(kept), C.byref(last))
    return n, kept.value, last.value


def kept_positions(src: bytes, pat: bytes, block_before: int = 0) -> list[int]:
    lib = _load()
    cap = len(src) // max(len(pat), 1) + 1
    arr = (C.c_int64 * cap)()
    k = lib.oracle_kept_positions(src, len(src), pat, len(pat), block_before, arr, cap)
    return list(arr[:k])


def query_prefix(src: bytes, pat: bytes, limit: int, block_before: int = 0) -> Tuple[int, int]:
    lib = _load()
    kept, last = C.c_int64(0), C.c_int64(-1)
    lib.oracle_query_prefix(src, len(src), pat, len(pat), block_before, limit, C.byref(kept), C.byref(last))
    return kept.value, last.value


def py_replace(src: bytes, pat: bytes, rep: bytes, block_before: int = 0) -> bytes:
    """Pure-Python restatement of the greedy (small inputs only)."""
    L = len(pat)
    if L == 0:
        return rep + b"".join(bytes([b]) + rep for b in src)
    out = bytearray()
    blocked = max(0, block_before)
    i = 0
    pos = 0  # first byte not yet emitted
    while i + L <= len(src):
        if i >= blocked and src[i:i + L] == pat:
            out += src[pos:i] + rep
            pos = i + L
            blocked = i + L
            i += L
        else:
            i += 1
    out += src[pos:]
    return bytes(out)


def bytes_replace(src: bytes, pat: bytes, rep: bytes) -> bytes:
    """The ground truth: CPython bytes.replace."""
    return src.replace(pat, rep)


def chain(src: bytes, pairs: Iterable[Tuple[bytes, bytes]]) -> bytes:
    """Sequential pairs, each applied to the previous output (apply_batch / streaming)."""
    out = src
    for pat, rep in pairs:
        out = out.replace(pat, rep)
    return out


def chain_lengths(src: bytes, pairs: Sequence[Tuple[bytes, bytes]]) -> list[int]:
    out, lens = src, [len(src)]
    for pat, rep in pairs:
        out = out.replace(pat, rep)
        lens.append(len(out))
    return lens
