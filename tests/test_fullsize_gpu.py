"""Full-size checks of the 2 GiB / 1 GiB single-pair configuration through the device-resident
entry point (cuda_replace_apply_device_async). Outputs too large to compare byte by byte
on the host are checked through size-independent properties on the device: exact output
length, periodicity of the replacement stream, and a SHA-256 against the C oracle where the
oracle finishes in seconds. torch only provides device memory and the comparisons."""
import hashlib

import numpy as np
import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu

GiB = 1 << 30


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _apply(sess, torch, d_in, n, pat, rep, cap):
    out = torch.empty(cap + 64, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    sess.apply_device_async(d_in.data_ptr(), n, pat, rep, out.data_ptr(), cap, stream)
    out_len, kept = sess.device_result()
    return out, out_len, kept


def test_run_2gib_aa_to_X(cr_lib, torch_cuda):
    torch = torch_cuda
    n = 2 * GiB
    d_in = torch.full((n + 64,), ord("a"), dtype=torch.uint8, device="cuda")
    with Wr.Session(cr_lib, b"") as s:
        out, out_len, kept = _apply(s, torch, d_in, n, b"aa", b"X", n)
    assert out_len == n // 2 and kept == n // 2
    assert bool((out[:out_len] == ord("X")).all())
    del out, d_in
    torch.cuda.empty_cache()


def test_run_2gib_a_to_bcd_64bit_offsets(cr_lib, torch_cuda):
    torch = torch_cuda
    n = 2 * GiB
    d_in = torch.full((n + 64,), ord("a"), dtype=torch.uint8, device="cuda")
    with Wr.Session(cr_lib, b"") as s:
        out, out_len, kept = _apply(s, torch, d_in, n, b"a", b"bcd", 3 * n)
    assert out_len == 3 * n and kept == n  # 6 GiB output: offsets beyond 2**32
    tri = out[:out_len].view(-1, 3)
    want = torch.tensor([ord("b"), ord("c"), ord("d")], dtype=torch.uint8, device="cuda")
    assert bool((tri == want).all())
    del out, tri, d_in
    torch.cuda.empty_cache()


def test_random_1gib_delete_nul_pattern(cr_lib, torch_cuda, oracle_mod):
    torch = torch_cuda
    name, gen, pat, rep = WL.c2_cases(n_rand=1 * GiB)[2]
    data = gen()
    n = len(data)
    host = np.frombuffer(data, dtype=np.uint8)
    d_in = torch.empty(n + 64, dtype=torch.uint8, device="cuda")
    d_in[:n].copy_(torch.from_numpy(host.copy()))
    with Wr.Session(cr_lib, b"") as s:
        out, out_len, kept = _apply(s, torch, d_in, n, pat, rep, n)
    got = out[:out_len].cpu().numpy().tobytes()
    exp, exp_kept, _ = oracle_mod.replace(data, pat, rep)
    assert out_len == len(exp) and kept == exp_kept
    assert hashlib.sha256(got).digest() == hashlib.sha256(exp).digest()


def test_session_chain_on_device_matches_oracle(cr_lib, torch_cuda):
    """Session apply (unsynchronised output sizing) on a 256 MiB text with the 128 pairs."""
    txt = WL.text_corpus(256 << 20, seed=3)
    pairs = WL.c3_pairs(seed=3)
    exp = txt
    for p, r in pairs:
        exp = exp.replace(p, r)
    with Wr.Session(cr_lib, txt) as s:
        n = s.apply_batch(pairs)
        out = s.result()
    assert n == len(exp) and out == exp
