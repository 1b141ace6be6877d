"""cuda_replace_apply_device_noalloc: the entry point for callers that cannot allocate memory
when they call (a pool or arena owns the device budget, or the host forbids cudaMalloc and
cudaFree because they can stall the device). Its output must equal that of the existing
device entry point, cuda_replace_apply_device_async, bit for bit, on two calls in a row
(the second call reuses the fixed scratch array left behind by the first). The file name
sorts last so a run that stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from cuda_replace_b200 import workloads as WL
from cuda_replace_b200.cuda_replace_wrapper import Session

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, d_in, n, pat, rep, cap):
    fn = lib.lib.cuda_replace_apply_device_noalloc
    fn.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p, C.c_int, C.c_char_p, C.c_int,
                   C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_void_p]
    fn.restype = C.c_int
    out = torch.empty(cap + 64, dtype=torch.uint8, device="cuda")
    out_len = C.c_size_t(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(d_in.data_ptr() if d_in is not None else None, n, pat, len(pat), rep, len(rep),
            out.data_ptr(), cap, C.byref(out_len), stream)
    return rc, out, out_len.value


def _existing(lib, torch, d_in, n, pat, rep, cap):
    out = torch.empty(cap + 64, dtype=torch.uint8, device="cuda")
    with Session(lib, b"") as s:
        s.apply_device_async(d_in.data_ptr(), n, pat, rep, out.data_ptr(), cap,
                             torch.cuda.current_stream().cuda_stream)
        out_len, _ = s.device_result()
    return out, out_len


def _device(torch, data: bytes):
    t = torch.empty(len(data) + 64, dtype=torch.uint8, device="cuda")
    t[:len(data)].copy_(torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()))
    return t


def test_noalloc_matches_existing_entry_point_twice(cr_lib):
    import torch
    assert torch.cuda.is_available()
    acgt, _, _ = WL.c1_acgt(16 << 20, seed=1)
    cases = [
        (b"a" * (5 * (1 << 20) + 3), b"aa", b"X"),   # bordered pattern: carry tables in the scratch
        (acgt, b"ACGT", b"N"),                       # borderless pattern: kept-count look-back
    ]
    for data, pat, rep in cases:  # two calls in a row on the same scratch array
        d_in = _device(torch, data)
        n = len(data)
        cap = n + (n // len(pat)) * max(0, len(rep) - len(pat))
        rc, got, got_len = _noalloc(cr_lib, torch, d_in, n, pat, rep, cap)
        assert rc == 0
        want, want_len = _existing(cr_lib, torch, d_in, n, pat, rep, cap)
        assert got_len == want_len == len(data.replace(pat, rep))
        assert bool((got[:got_len] == want[:want_len]).all())


def test_noalloc_rejects_sizes_beyond_its_limits(cr_lib):
    import torch
    d_in = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    rc, _, _ = _noalloc(cr_lib, torch, d_in, (64 << 20) + 1, b"ab", b"", (64 << 20) + 1)
    assert rc == -6
    rc, _, _ = _noalloc(cr_lib, torch, d_in, 512, b"p" * 65, b"", 512)
    assert rc == -6


def test_noalloc_at_its_size_limit_and_without_allocating(cr_lib):
    """At the largest input the fixed scratch holds (every tile slot used) with a 64-byte
    pattern that has a border (so each tile stores its full table of 64 carry entries): the
    output equals bytes.replace and the existing entry point, on two calls in a row, and a
    warm call leaves the device's free memory unchanged."""
    import torch
    n = 64 << 20
    unit = b"ab" * 40 + b"x" + b"ab" * 31 + b"y"  # full and near matches of (ab)*32
    data = (unit * (n // len(unit) + 1))[:n]
    pat, rep = b"ab" * 32, b"Q"
    d_in = _device(torch, data)
    want = data.replace(pat, rep)
    for _ in range(2):
        rc, got, got_len = _noalloc(cr_lib, torch, d_in, n, pat, rep, n)
        assert rc == 0 and got_len == len(want)
        assert bytes(got[:got_len].cpu().numpy()) == want
    ref, ref_len = _existing(cr_lib, torch, d_in, n, pat, rep, n)
    assert ref_len == got_len and bool((ref[:ref_len] == got[:got_len]).all())
    out = torch.empty(n + 64, dtype=torch.uint8, device="cuda")
    fn = cr_lib.lib.cuda_replace_apply_device_noalloc
    out_len = C.c_size_t(0)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = fn(d_in.data_ptr(), n, pat, len(pat), rep, len(rep), out.data_ptr(), n, C.byref(out_len), stream)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0 and out_len.value == len(want)
    assert free_after == free_before
