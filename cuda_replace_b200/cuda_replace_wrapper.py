"""ctypes binding of libcuda_replace.so with the interface of the reference wrapper.

Same names, arguments, return values and errors as RAZZULLIX/cuda_replace's
cuda_replace_wrapper.py (``CudaReplaceLib.unified`` py:124-141, ``Session`` py:145-297,
``replace_unified`` py:301-303, ``gpu_replace_streaming`` py:305-366), so code written
against the reference runs unchanged. Every call goes to the CUDA library; there is no CPU
path, and loading fails loudly when the library has not been built.

``gpu_replace_streaming`` keeps its signature but not the reference body: the reference
cuts each chunk's output at ``(base_end-pos) + kept_before*diff`` (py:356), which drops the
replacement of a match that straddles the chunk boundary and re-emits the bytes it covers.
The version here cuts after that replacement and drops the covered bytes at the start of
the next chunk, so the result equals the chained ``bytes.replace`` for any chunk size.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Iterable, List, Optional, Sequence, Tuple

_PKG_DIR = Path(__file__).resolve().parent
DEFAULT_LIB = _PKG_DIR / "libcuda_replace.so"

c_size_t = C.c_size_t
c_uint8_p = C.POINTER(C.c_uint8)
c_void_p = C.c_void_p
c_int_p = C.POINTER(C.c_int)
c_longlong_p = C.POINTER(C.c_longlong)
c_size_t_p = C.POINTER(c_size_t)
c_uint8_pp = C.POINTER(c_uint8_p)


_new_bytes = C.pythonapi.PyBytes_FromStringAndSize
_new_bytes.restype = C.py_object
_new_bytes.argtypes = [C.c_void_p, C.c_ssize_t]
_bytes_buffer = C.pythonapi.PyBytes_AsString
_bytes_buffer.restype = C.c_void_p
_bytes_buffer.argtypes = [C.py_object]
_PARALLEL_COPY_MIN = 4 << 20
# The same calls with raw object pointers (new function objects: pythonapi caches the ones
# above by attribute), for a bytes object filled and shrunk before Python code sees it.
_new_bytes_raw = C.pythonapi["PyBytes_FromStringAndSize"]
_new_bytes_raw.restype = C.c_void_p
_new_bytes_raw.argtypes = [C.c_void_p, C.c_ssize_t]
_raw_buffer = C.pythonapi["PyBytes_AsString"]
_raw_buffer.restype = C.c_void_p
_raw_buffer.argtypes = [C.c_void_p]
_raw_resize = C.pythonapi["_PyBytes_Resize"]
_raw_resize.restype = C.c_int
_raw_resize.argtypes = [C.POINTER(C.c_void_p), C.c_ssize_t]
_raw_decref = C.pythonapi["Py_DecRef"]
_raw_decref.restype = None
_raw_decref.argtypes = [C.c_void_p]


def _bytes_filled(n: int, fill) -> bytes:
    """A bytes object of at most n bytes written by fill(address, n) -> length: created
    uninitialised at n bytes, filled in place (no second copy of the result), then shrunk to
    the length written (a realloc that large blocks do in place). The object is private to this
    function until it returns, so resizing it is allowed (_PyBytes_Resize needs one reference)."""
    raw = _new_bytes_raw(None, n)
    if not raw:
        raise MemoryError(f"bytes object of {n} bytes")
    try:
        addr = _raw_buffer(raw)
        _advise_huge(addr, n)
        m = fill(addr, n)
    except BaseException:
        _raw_decref(raw)
        raise
    box = c_void_p(raw)
    if m != n:
        _raw_resize(C.byref(box), m)  # raises MemoryError (object freed) if it fails
    out = C.cast(box, C.py_object).value  # a new reference ...
    _raw_decref(box)                      # ... and the creation's released
    return out


def _bytes_at(ptr, n: int, lib: Optional[C.CDLL] = None) -> bytes:
    """Copy n bytes of library-owned memory into a new bytes object. Large results are copied
    by the library on several host threads into a bytes object created uninitialised (the
    page faults of fresh memory, not the copy, bound a single-threaded copy); ctypes.string_at
    is not used because its size is a C int, which results of 2 GiB and more overflow."""
    if not n:
        return b""
    addr = C.cast(ptr, c_void_p).value
    copy = getattr(lib, "cuda_replace_host_copy", None) if lib is not None else None
    if copy is None or n < _PARALLEL_COPY_MIN:
        return memoryview((C.c_uint8 * n).from_address(addr)).cast("B").tobytes()
    out = _new_bytes(None, n)  # uninitialised, filled below before anyone else sees it
    dst = _bytes_buffer(out)
    _advise_huge(dst, n)
    copy(c_void_p(dst), c_void_p(addr), c_size_t(n))
    return out


_MADV_HUGEPAGE = 14
try:
    _libc = C.CDLL(None, use_errno=True)
    _madvise = _libc.madvise
    _madvise.argtypes = [c_void_p, c_size_t, C.c_int]
    _madvise.restype = C.c_int
except (OSError, AttributeError):
    _madvise = None


def _advise_huge(addr: int, n: int) -> None:
    """Ask for 2 MiB pages on the whole 2 MiB blocks of a fresh result buffer: the first touch
    of gigabytes of 4 KiB pages (one fault and one zeroing per page) bounds the copy out of the
    library's page-locked block otherwise. Only a hint; ignored where not supported."""
    if _madvise is None or n < (64 << 20):
        return
    a = (addr + (2 << 20) - 1) & ~((2 << 20) - 1)
    e = (addr + n) & ~((2 << 20) - 1)
    if e > a:
        _madvise(c_void_p(a), c_size_t(e - a), C.c_int(_MADV_HUGEPAGE))


def _src_pointer(src):
    """(keep-alive object, pointer, length) of a bytes-like input without copying bytes objects."""
    if isinstance(src, bytes):
        return src, (C.cast(C.c_char_p(src), c_uint8_p) if src else c_uint8_p()), len(src)
    mv = memoryview(src)
    n = mv.nbytes
    if not n:
        return None, c_uint8_p(), 0
    if mv.readonly:
        b = bytes(mv)
        return b, C.cast(C.c_char_p(b), c_uint8_p), n
    holder = (C.c_uint8 * n).from_buffer(mv)
    return holder, C.cast(holder, c_uint8_p), n


def _bind(lib: C.CDLL, name: str, argtypes, restype, optional: bool = False) -> None:
    if optional and not hasattr(lib, name):
        setattr(lib, name, None)  # additive entry point absent from this build
        return
    fn = getattr(lib, name)
    fn.argtypes = argtypes
    fn.restype = restype


class ServerStats(C.Structure):
    """CudaReplaceServerStats (include/cuda_replace.h)."""
    _fields_ = [("jobs_done", C.c_ulonglong), ("jobs_via_session", C.c_ulonglong), ("batches", C.c_ulonglong),
                ("bytes_in", C.c_ulonglong), ("bytes_out", C.c_ulonglong), ("kernel_launches", C.c_ulonglong),
                ("graph_launches", C.c_ulonglong), ("pending", C.c_ulonglong), ("arena_bytes", C.c_ulonglong),
                ("arena_peak_bytes", C.c_ulonglong), ("p50_us", C.c_double), ("p99_us", C.c_double),
                ("max_us", C.c_double), ("gpu_us", C.c_double), ("download_us", C.c_double),
                ("session_us", C.c_double), ("tile_bytes", C.c_uint * 3), ("grid_ctas", C.c_int * 3),
                ("cancelled", C.c_ulonglong)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["tile_bytes"] = list(self.tile_bytes)
        d["grid_ctas"] = list(self.grid_ctas)
        return d


class CudaReplaceLib:
    """Loads libcuda_replace.so and binds its C ABI (reference: py:36-141)."""

    def __init__(self, dll_path: Optional[str] = None):
        path = Path(os.fspath(dll_path)) if dll_path else DEFAULT_LIB
        if not path.exists():
            raise FileNotFoundError(
                f"{path} not found: build it with `python -m cuda_replace_b200.build` "
                "(the replace path has no CPU fallback)")
        self.path = str(path)
        self.lib = C.CDLL(self.path, use_errno=True)
        lib = self.lib
        _bind(lib, "cuda_replace_unified",
              [c_uint8_p, c_size_t, c_uint8_p, C.c_int, c_uint8_p, C.c_int, C.POINTER(c_uint8_p), c_size_t_p],
              C.c_int)
        _bind(lib, "cuda_free_host", [c_void_p], None)
        _bind(lib, "cuda_replace_open", [C.POINTER(c_void_p), c_uint8_p, c_size_t], C.c_int)
        _bind(lib, "cuda_replace_build_index", [c_void_p, c_size_t], C.c_int)
        _bind(lib, "cuda_replace_apply", [c_void_p, c_uint8_p, C.c_int, c_uint8_p, C.c_int, c_size_t_p], C.c_int)
        _bind(lib, "cuda_replace_apply_batch",
              [c_void_p, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int, c_size_t_p], C.c_int)
        _bind(lib, "cuda_replace_result", [c_void_p, C.POINTER(c_uint8_p), c_size_t_p], C.c_int)
        _bind(lib, "cuda_replace_close", [c_void_p], None)
        _bind(lib, "cuda_replace_reset", [c_void_p, c_uint8_p, c_size_t], C.c_int)
        _bind(lib, "cuda_replace_apply_seeded",
              [c_void_p, c_uint8_p, C.c_int, c_uint8_p, C.c_int, C.c_longlong, c_longlong_p, c_size_t_p],
              C.c_int)
        _bind(lib, "cuda_replace_query_prefix", [c_void_p, c_size_t, c_int_p, c_int_p], C.c_int)
        _bind(lib, "cuda_replace_version", [], C.c_char_p)
        # additive entry points
        _bind(lib, "cuda_replace_length", [c_void_p, c_size_t_p], C.c_int)
        _bind(lib, "cuda_replace_query_prefix64", [c_void_p, c_size_t, c_longlong_p, c_longlong_p], C.c_int)
        _bind(lib, "cuda_replace_result_into", [c_void_p, c_void_p, c_size_t, c_size_t_p], C.c_int)
        _bind(lib, "cuda_replace_stats",
              [c_void_p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)], C.c_int)
        _bind(lib, "cuda_replace_apply_device_async",
              [c_void_p, c_void_p, c_size_t, c_uint8_p, C.c_int, c_uint8_p, C.c_int, c_void_p, c_size_t, c_void_p],
              C.c_int, optional=True)
        _bind(lib, "cuda_replace_device_result", [c_void_p, c_size_t_p, C.POINTER(C.c_ulonglong)], C.c_int,
              optional=True)
        _bind(lib, "cuda_replace_server_open", [C.POINTER(c_void_p), c_size_t, C.c_int], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_submit",
              [c_void_p, c_uint8_p, c_size_t, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int,
               C.POINTER(C.c_ulonglong)], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_submit_tenant",
              [c_void_p, C.c_uint, c_uint8_p, c_size_t, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int,
               C.POINTER(C.c_ulonglong)], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_cancel", [c_void_p, C.c_ulonglong], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_set_tenant_budget", [c_void_p, C.c_uint, c_size_t], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_tenant_usage",
              [c_void_p, C.c_uint, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_wait",
              [c_void_p, C.c_ulonglong, C.c_int, C.POINTER(c_uint8_p), c_size_t_p], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_stats", [c_void_p, C.POINTER(ServerStats)], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_reset_stats", [c_void_p], C.c_int, optional=True)
        _bind(lib, "cuda_replace_server_close", [c_void_p], None, optional=True)
        _bind(lib, "cuda_replace_jobs",
              [C.c_int, c_uint8_pp, c_size_t_p, c_int_p, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p,
               c_uint8_pp, c_size_t_p], C.c_int, optional=True)
        _bind(lib, "cuda_replace_jobs_release", [], None, optional=True)
        _bind(lib, "cuda_replace_stream_fd",
              [C.c_int, C.c_int, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int, c_size_t,
               C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)], C.c_int, optional=True)
        _bind(lib, "cuda_replace_plan_stages",
              [c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int, C.c_int, c_int_p], C.c_int, optional=True)
        _bind(lib, "cuda_replace_host_copy", [c_void_p, c_void_p, c_size_t], None, optional=True)
        _bind(lib, "cuda_replace_unified_into",
              [c_uint8_p, c_size_t, c_uint8_p, C.c_int, c_uint8_p, C.c_int, c_void_p, c_size_t, c_size_t_p], C.c_int,
              optional=True)
        _bind(lib, "cuda_replace_output_bound", [c_size_t, C.c_int, C.c_int, c_size_t_p], C.c_int, optional=True)
        _bind(lib, "cuda_replace_stream",
              [c_uint8_p, c_size_t, c_uint8_pp, c_int_p, c_uint8_pp, c_int_p, C.c_int, c_size_t,
               C.POINTER(c_uint8_p), c_size_t_p], C.c_int, optional=True)

    def version(self) -> str:
        return self.lib.cuda_replace_version().decode()

    def unified(self, src: bytes, pat: bytes, rep: bytes) -> bytes:
        """One-shot replace (reference: py:124-141). A large result is written straight into the
        returned bytes object (cuda_replace_unified_into): its copy out of page-locked memory
        overlaps the transfers instead of following them."""
        keep, src_p, n = _src_pointer(src)
        pat_buf = C.create_string_buffer(pat, len(pat) or 1)
        rep_buf = C.create_string_buffer(rep, len(rep) or 1)
        into = getattr(self.lib, "cuda_replace_unified_into", None)
        if into is not None and pat and n >= _PARALLEL_COPY_MIN:
            bound = c_size_t()
            self.lib.cuda_replace_output_bound(c_size_t(n), C.c_int(len(pat)), C.c_int(len(rep)), C.byref(bound))
            if bound.value <= 4 * n + (64 << 20):
                def fill(addr, cap):
                    got = c_size_t()
                    rc = into(src_p, c_size_t(n), C.cast(pat_buf, c_uint8_p), C.c_int(len(pat)),
                              C.cast(rep_buf, c_uint8_p), C.c_int(len(rep)), c_void_p(addr), c_size_t(cap),
                              C.byref(got))
                    if rc != 0:
                        raise RuntimeError(f"cuda_replace_unified_into failed rc={rc}")
                    return got.value
                try:
                    return _bytes_filled(bound.value, fill)
                finally:
                    del keep
        out_ptr = c_uint8_p()
        out_len = c_size_t()
        rc = self.lib.cuda_replace_unified(
            src_p, c_size_t(n),
            C.cast(pat_buf, c_uint8_p), C.c_int(len(pat)),
            C.cast(rep_buf, c_uint8_p), C.c_int(len(rep)),
            C.byref(out_ptr), C.byref(out_len))
        del keep
        if rc != 0:
            raise RuntimeError(f"cuda_replace_unified failed rc={rc}")
        try:
            return _bytes_at(out_ptr, out_len.value, self.lib)
        finally:
            self.lib.cuda_free_host(out_ptr)


class Session:
    """A device-resident buffer that successive replaces transform in place (reference: py:145-297)."""

    def __init__(self, lib: CudaReplaceLib, src: bytes):
        self.lib = lib
        self.h = c_void_p()
        keep, src_p, n = _src_pointer(src)
        rc = lib.lib.cuda_replace_open(C.byref(self.h), src_p, c_size_t(n))
        del keep
        if rc != 0:
            raise RuntimeError(f"cuda_replace_open failed rc={rc}")

    def __enter__(self) -> "Session":
        return self

    def __exit__(self, exc_type, exc, tb):
        self.close()

    def reset(self, src: bytes) -> None:
        keep, src_p, n = _src_pointer(src)
        rc = self.lib.lib.cuda_replace_reset(self.h, src_p, c_size_t(n))
        del keep
        if rc != 0:
            raise RuntimeError(f"cuda_replace_reset failed rc={rc}")

    def build_index(self, chunk_size: Optional[int] = None) -> None:
        rc = self.lib.lib.cuda_replace_build_index(self.h, c_size_t(0 if chunk_size is None else int(chunk_size)))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_build_index failed rc={rc}")

    def apply(self, pat: bytes, rep: bytes) -> int:
        pb = C.create_string_buffer(pat, len(pat) or 1)
        rb = C.create_string_buffer(rep, len(rep) or 1)
        new_len = c_size_t()
        rc = self.lib.lib.cuda_replace_apply(self.h, C.cast(pb, c_uint8_p), C.c_int(len(pat)),
                                             C.cast(rb, c_uint8_p), C.c_int(len(rep)), C.byref(new_len))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_apply failed rc={rc}")
        return int(new_len.value)

    def apply_seeded(self, pat: bytes, rep: bytes, prev_last_rel: int) -> Tuple[int, int]:
        """Apply with carry-in; returns (new_len, last kept start in this buffer or -1)."""
        pb = C.create_string_buffer(pat, len(pat) or 1)
        rb = C.create_string_buffer(rep, len(rep) or 1)
        new_len = c_size_t()
        last = C.c_longlong(-1)
        rc = self.lib.lib.cuda_replace_apply_seeded(
            self.h, C.cast(pb, c_uint8_p), C.c_int(len(pat)), C.cast(rb, c_uint8_p), C.c_int(len(rep)),
            C.c_longlong(int(prev_last_rel)), C.byref(last), C.byref(new_len))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_apply_seeded failed rc={rc}")
        return int(new_len.value), int(last.value)

    def apply_batch(self, pairs: Sequence[Tuple[bytes, bytes]]) -> int:
        count = len(pairs)
        if count == 0:
            return self.length()
        keep = []
        pat_ptrs = (c_uint8_p * count)()
        rep_ptrs = (c_uint8_p * count)()
        pat_lens = (C.c_int * count)()
        rep_lens = (C.c_int * count)()
        for i, (pat, rep) in enumerate(pairs):
            pb = C.create_string_buffer(pat, len(pat) or 1)
            rb = C.create_string_buffer(rep, len(rep) or 1)
            keep += [pb, rb]
            pat_ptrs[i] = C.cast(pb, c_uint8_p)
            rep_ptrs[i] = C.cast(rb, c_uint8_p)
            pat_lens[i] = len(pat)
            rep_lens[i] = len(rep)
        new_len = c_size_t()
        rc = self.lib.lib.cuda_replace_apply_batch(
            self.h, C.cast(pat_ptrs, c_uint8_pp), C.cast(pat_lens, c_int_p),
            C.cast(rep_ptrs, c_uint8_pp), C.cast(rep_lens, c_int_p), C.c_int(count), C.byref(new_len))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_apply_batch failed rc={rc}")
        return int(new_len.value)

    def query_prefix(self, limit: int) -> Tuple[int, int]:
        """(kept starts before limit, last such start or -1) of the most recent apply."""
        kept = C.c_longlong(0)
        last = C.c_longlong(-1)
        rc = self.lib.lib.cuda_replace_query_prefix64(self.h, c_size_t(int(limit)), C.byref(kept), C.byref(last))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_query_prefix failed rc={rc}")
        return int(kept.value), int(last.value)

    def result(self) -> bytes:
        out_ptr = c_uint8_p()
        out_len = c_size_t()
        rc = self.lib.lib.cuda_replace_result(self.h, C.byref(out_ptr), C.byref(out_len))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_result failed rc={rc}")
        try:
            return _bytes_at(out_ptr, out_len.value, self.lib.lib)
        finally:
            self.lib.lib.cuda_free_host(out_ptr)

    def length(self) -> int:
        n = c_size_t()
        rc = self.lib.lib.cuda_replace_length(self.h, C.byref(n))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_length failed rc={rc}")
        return int(n.value)

    def stats(self) -> Tuple[int, int]:
        kept, launches = C.c_ulonglong(0), C.c_ulonglong(0)
        rc = self.lib.lib.cuda_replace_stats(self.h, C.byref(kept), C.byref(launches))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_stats failed rc={rc}")
        return int(kept.value), int(launches.value)

    def apply_device_async(self, d_in: int, n: int, pat: bytes, rep: bytes, d_out: int, out_cap: int,
                           stream: int = 0) -> None:
        """Enqueue a replace of device memory d_in[0, n) into d_out on a CUDA stream handle."""
        pb = C.create_string_buffer(pat, len(pat) or 1)
        rb = C.create_string_buffer(rep, len(rep) or 1)
        rc = self.lib.lib.cuda_replace_apply_device_async(
            self.h, c_void_p(d_in), c_size_t(n), C.cast(pb, c_uint8_p), C.c_int(len(pat)),
            C.cast(rb, c_uint8_p), C.c_int(len(rep)), c_void_p(d_out), c_size_t(out_cap), c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_apply_device_async failed rc={rc}")

    def device_result(self) -> Tuple[int, int]:
        """(output length, matches kept) of the last apply_device_async, after waiting for it."""
        n, kept = c_size_t(0), C.c_ulonglong(0)
        rc = self.lib.lib.cuda_replace_device_result(self.h, C.byref(n), C.byref(kept))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_device_result failed rc={rc}")
        return int(n.value), int(kept.value)

    def close(self) -> None:
        if self.h:
            self.lib.lib.cuda_replace_close(self.h)
            self.h = c_void_p(None)


class CancelledJob(Exception):
    """Server.wait on a job that Server.cancel removed from the queue."""


class Server:
    """Request loop over batched segmented launches (no counterpart in the reference).

    ``submit(data, pairs)`` queues a job (its input and its own sequence of pairs) and returns
    a ticket; ``wait(ticket)`` returns the job's result, equal to the chained bytes.replace.
    Jobs that arrive while a batch is on the GPU are admitted to the next batch as device
    memory (``hbm_budget`` bytes, 0 = 40% of the free memory) and one of two batch slots free
    up; ``stats()`` reports throughput and p50/p99 latency from submit to result."""

    def __init__(self, lib: CudaReplaceLib, hbm_budget: int = 0, max_jobs_per_batch: int = 0):
        if getattr(lib.lib, "cuda_replace_server_open", None) is None:
            raise RuntimeError("this libcuda_replace.so has no server entry points")
        self.lib = lib
        self.h = c_void_p()
        rc = lib.lib.cuda_replace_server_open(C.byref(self.h), c_size_t(int(hbm_budget)), C.c_int(max_jobs_per_batch))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_server_open failed rc={rc}")

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, exc_type, exc, tb):
        self.close()

    def submit(self, data, pairs: Sequence[Tuple[bytes, bytes]], tenant: int = 0) -> int:
        """Queue a job; tenant >= 1 counts its device memory against that tenant's budget."""
        keep, pat_ptrs, pat_lens, rep_ptrs, rep_lens = _pair_arrays(pairs)
        holder, src_ptr, n = _src_pointer(data)
        ticket = C.c_ulonglong(0)
        args = (src_ptr, c_size_t(n), C.cast(pat_ptrs, c_uint8_pp), C.cast(pat_lens, c_int_p),
                C.cast(rep_ptrs, c_uint8_pp), C.cast(rep_lens, c_int_p), C.c_int(len(pairs)), C.byref(ticket))
        if tenant:
            rc = self.lib.lib.cuda_replace_server_submit_tenant(self.h, C.c_uint(tenant), *args)
        else:
            rc = self.lib.lib.cuda_replace_server_submit(self.h, *args)
        del keep, holder
        if rc == -9:
            raise MemoryError(f"the job needs more device memory than tenant {tenant}'s budget")
        if rc != 0:
            raise RuntimeError(f"cuda_replace_server_submit failed rc={rc}")
        return int(ticket.value)

    def cancel(self, ticket: int) -> bool:
        """True when the job was still queued and is cancelled (its wait then raises
        CancelledJob); False when it is already on the device or done (it completes normally)."""
        rc = self.lib.lib.cuda_replace_server_cancel(self.h, C.c_ulonglong(ticket))
        if rc < 0:
            raise KeyError(ticket)
        return rc == 0

    def set_tenant_budget(self, tenant: int, nbytes: int) -> None:
        """Device memory that tenant's jobs may hold at once (0: no limit)."""
        rc = self.lib.lib.cuda_replace_server_set_tenant_budget(self.h, C.c_uint(tenant), c_size_t(int(nbytes)))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_server_set_tenant_budget failed rc={rc}")

    def tenant_usage(self, tenant: int) -> Tuple[int, int]:
        """(bytes the tenant's jobs hold on the device now, the most they held at once)."""
        cur, peak = C.c_ulonglong(0), C.c_ulonglong(0)
        self.lib.lib.cuda_replace_server_tenant_usage(self.h, C.c_uint(tenant), C.byref(cur), C.byref(peak))
        return int(cur.value), int(peak.value)

    def wait(self, ticket: int, timeout_ms: int = -1) -> Optional[bytes]:
        """The job's result; None when it is not done within timeout_ms (negative: no limit)."""
        out_ptr = c_uint8_p()
        out_len = c_size_t()
        rc = self.lib.lib.cuda_replace_server_wait(self.h, C.c_ulonglong(ticket), C.c_int(timeout_ms),
                                                   C.byref(out_ptr), C.byref(out_len))
        if rc == 1:
            return None
        if rc == -8:
            raise CancelledJob(ticket)
        if rc != 0:
            raise RuntimeError(f"cuda_replace_server_wait failed rc={rc}")
        try:
            return _bytes_at(out_ptr, out_len.value, self.lib.lib)
        finally:
            self.lib.lib.cuda_free_host(out_ptr)

    def stats(self) -> dict:
        st = ServerStats()
        rc = self.lib.lib.cuda_replace_server_stats(self.h, C.byref(st))
        if rc != 0:
            raise RuntimeError(f"cuda_replace_server_stats failed rc={rc}")
        return st.as_dict()

    def reset_stats(self) -> None:
        self.lib.lib.cuda_replace_server_reset_stats(self.h)

    def close(self) -> None:
        if self.h:
            self.lib.lib.cuda_replace_server_close(self.h)
            self.h = c_void_p(None)


def replace_jobs(lib: CudaReplaceLib, jobs: Sequence[Tuple[bytes, Sequence[Tuple[bytes, bytes]]]]) -> List[bytes]:
    """Many independent jobs (input, pairs) in one call: each result equals the chained
    bytes.replace of its job. Runs as batched segmented launches (cuda_replace_jobs)."""
    fn = getattr(lib.lib, "cuda_replace_jobs", None)
    if fn is None:
        raise RuntimeError("this libcuda_replace.so has no cuda_replace_jobs")
    nj = len(jobs)
    if nj == 0:
        return []
    srcs = (c_uint8_p * nj)()
    lens = (c_size_t * nj)()
    counts = (C.c_int * nj)()
    flat: List[Tuple[bytes, bytes]] = []
    holders = []
    for i, (data, pairs) in enumerate(jobs):
        b = data if isinstance(data, bytes) else bytes(data)
        holders.append(b)
        srcs[i] = C.cast(C.c_char_p(b), c_uint8_p) if b else c_uint8_p()
        lens[i] = len(b)
        counts[i] = len(pairs)
        flat.extend(pairs)
    keep, pat_ptrs, pat_lens, rep_ptrs, rep_lens = _pair_arrays(flat)
    outs = (c_uint8_p * nj)()
    out_lens = (c_size_t * nj)()
    rc = fn(C.c_int(nj), C.cast(srcs, c_uint8_pp), C.cast(lens, c_size_t_p), C.cast(counts, c_int_p),
            C.cast(pat_ptrs, c_uint8_pp), C.cast(pat_lens, c_int_p), C.cast(rep_ptrs, c_uint8_pp),
            C.cast(rep_lens, c_int_p), C.cast(outs, c_uint8_pp), C.cast(out_lens, c_size_t_p))
    del keep, holders
    if rc != 0:
        raise RuntimeError(f"cuda_replace_jobs failed rc={rc}")
    res = []
    for i in range(nj):
        res.append(_bytes_at(outs[i], out_lens[i], lib.lib))
        lib.lib.cuda_free_host(outs[i])
    return res


def replace_unified(lib: CudaReplaceLib, src: bytes, pat: bytes, rep: bytes) -> bytes:
    """One-shot convenience around cuda_replace_unified (reference: py:301-303)."""
    return lib.unified(src, pat, rep)


def stream_chunk_plan(n: int, chunk_bytes: int) -> List[Tuple[int, int]]:
    """[pos, base_end) ranges of the chunks of an n-byte input."""
    chunk_bytes = max(1, int(chunk_bytes))
    return [(p, min(p + chunk_bytes, n)) for p in range(0, n, chunk_bytes)]


STREAM_UNSUPPORTED = -7  # cuda_replace_stream: a pair outside its limits


def _pair_arrays(pairs: Sequence[Tuple[bytes, bytes]]):
    count = max(len(pairs), 1)
    keep = []
    pat_ptrs = (c_uint8_p * count)()
    rep_ptrs = (c_uint8_p * count)()
    pat_lens = (C.c_int * count)()
    rep_lens = (C.c_int * count)()
    for i, (pat, rep) in enumerate(pairs):
        pb = C.create_string_buffer(pat, len(pat) or 1)
        rb = C.create_string_buffer(rep, len(rep) or 1)
        keep += [pb, rb]
        pat_ptrs[i] = C.cast(pb, c_uint8_p)
        rep_ptrs[i] = C.cast(rb, c_uint8_p)
        pat_lens[i] = len(pat)
        rep_lens[i] = len(rep)
    return keep, pat_ptrs, pat_lens, rep_ptrs, rep_lens


def stream_native(lib: CudaReplaceLib, src, pairs: Sequence[Tuple[bytes, bytes]],
                  chunk_bytes: int) -> Optional[bytes]:
    """Chunk-major streaming through cuda_replace_stream: every pair is applied to a chunk on
    the device before the next chunk is read. None when the library lacks the entry point or
    a pair is outside its limits (pattern 1-256 bytes, bordered patterns up to 32 bytes,
    replacement up to 256 bytes)."""
    fn = getattr(lib.lib, "cuda_replace_stream", None)
    if fn is None:
        return None
    keep, pat_ptrs, pat_lens, rep_ptrs, rep_lens = _pair_arrays(pairs)
    holder, src_ptr, n = _src_pointer(src)
    out_ptr = c_uint8_p()
    out_len = c_size_t()
    rc = fn(src_ptr, c_size_t(n), C.cast(pat_ptrs, c_uint8_pp), C.cast(pat_lens, c_int_p),
            C.cast(rep_ptrs, c_uint8_pp), C.cast(rep_lens, c_int_p), C.c_int(len(pairs)),
            c_size_t(int(chunk_bytes)), C.byref(out_ptr), C.byref(out_len))
    del keep, holder
    if rc == STREAM_UNSUPPORTED:
        return None
    if rc != 0:
        raise RuntimeError(f"cuda_replace_stream failed rc={rc}")
    try:
        return _bytes_at(out_ptr, out_len.value, lib.lib)
    finally:
        lib.lib.cuda_free_host(out_ptr)


def stream_file(lib: CudaReplaceLib, in_fd: int, out_fd: int, pairs: Sequence[Tuple[bytes, bytes]],
                chunk_bytes: int = 256 * 1024 * 1024) -> Tuple[int, int]:
    """Chained replacement from one open file descriptor to another (cuda_replace_stream_fd):
    chunk-major on the device, the input read and the output written piece by piece, so
    neither is held whole in memory. Returns (bytes read, bytes written)."""
    fn = getattr(lib.lib, "cuda_replace_stream_fd", None)
    if fn is None:
        raise RuntimeError("this libcuda_replace.so has no cuda_replace_stream_fd")
    keep, pat_ptrs, pat_lens, rep_ptrs, rep_lens = _pair_arrays(pairs)
    nin, nout = C.c_ulonglong(0), C.c_ulonglong(0)
    rc = fn(C.c_int(in_fd), C.c_int(out_fd), C.cast(pat_ptrs, c_uint8_pp), C.cast(pat_lens, c_int_p),
            C.cast(rep_ptrs, c_uint8_pp), C.cast(rep_lens, c_int_p), C.c_int(len(pairs)),
            c_size_t(int(chunk_bytes)), C.byref(nin), C.byref(nout))
    del keep
    if rc == STREAM_UNSUPPORTED:
        raise ValueError("a pair is outside the limits of the chunk-major stream")
    if rc == -10:
        raise OSError(C.get_errno(), "cuda_replace_stream_fd: reading or writing failed")
    if rc != 0:
        raise RuntimeError(f"cuda_replace_stream_fd failed rc={rc}")
    return int(nin.value), int(nout.value)


def _stream_supported(lib: CudaReplaceLib, pat: bytes, rep: bytes) -> bool:
    """Whether cuda_replace_stream takes this pair (asked with an empty input)."""
    return getattr(lib.lib, "cuda_replace_stream", None) is not None and \
        stream_native(lib, b"", [(pat, rep)], 1) is not None


def gpu_replace_streaming(lib: CudaReplaceLib, src: bytes, pairs: Iterable[Tuple[bytes, bytes]],
                          chunk_bytes: int = 256 * 1024 * 1024) -> bytes:
    """Chunked replacement of an input larger than device memory (reference signature:
    py:305-308). Runs of consecutive pairs that cuda_replace_stream takes go through it
    chunk-major; any other pair is streamed pair-major: each chunk carries an (L-1)-byte
    halo, and the carry-in is the start of the previous chunk's last kept match, passed to
    apply_seeded."""
    pairs = list(pairs)
    out = src
    i = 0
    while i < len(pairs):
        j = i
        while j < len(pairs) and _stream_supported(lib, *pairs[j]):
            j += 1
        if j > i:
            res = stream_native(lib, out, pairs[i:j], chunk_bytes)
            if res is None:
                raise RuntimeError("cuda_replace_stream rejected pairs it accepted alone")
            out, i = res, j
        else:
            out = _stream_pair_major(lib, out, pairs[i], chunk_bytes)
            i += 1
    return out


def _stream_pair_major(lib: CudaReplaceLib, src: bytes, pair: Tuple[bytes, bytes], chunk_bytes: int) -> bytes:
    out = src
    with Session(lib, b"") as sess:
        for pat, rep in [pair]:
            L = len(pat)
            n = len(out)
            pieces: List[bytes] = []
            if L == 0:
                # bytes.replace(b"", rep): rep before each byte and once at the end
                plan = stream_chunk_plan(n, chunk_bytes)
                for pos, base_end in plan:
                    sess.reset(out[pos:base_end])
                    sess.apply(pat, rep)
                    piece = sess.result()
                    pieces.append(piece[:len(piece) - len(rep)])
                pieces.append(rep)
                out = b"".join(pieces)
                continue
            diff = len(rep) - L
            prev_last: Optional[int] = None  # global start of the last kept match so far
            for pos, base_end in stream_chunk_plan(n, chunk_bytes):
                take_end = min(base_end + L - 1, n)
                sess.reset(out[pos:take_end])
                seed = (prev_last - pos) if prev_last is not None else -(1 << 62)
                sess.apply_seeded(pat, rep, seed)
                limit = base_end - pos
                kept_before, last_before = sess.query_prefix(limit)
                chunk_out = sess.result()
                # bytes covered by the previous chunk's last match were emitted as literals: drop
                skip = max(0, prev_last + L - pos) if prev_last is not None else 0
                overhang = max(0, last_before + L - limit) if kept_before else 0
                end = limit + kept_before * diff + overhang
                pieces.append(chunk_out[skip:end] if skip < end else b"")
                if kept_before:
                    prev_last = pos + last_before
            out = b"".join(pieces)
    return out
