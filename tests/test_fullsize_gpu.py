"""Full-size checks of the 2 GiB / 1 GiB single-pair configuration through the device-resident
entry point (cuda_replace_apply_device_async). Outputs too large to compare byte by byte
on the host are checked through size-independent properties on the device: exact output
length, periodicity of the replacement stream, and a SHA-256 against the C oracle where the
oracle finishes in seconds. torch only provides device memory and the comparisons."""
import hashlib
from pathlib import Path

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


# ------------------------------------------------------------------ full stated sizes
FULLSIZE = Path(__file__).parent / "golden" / "fullsize.json"


def _fullsize(key):
    import json
    if not FULLSIZE.exists():
        pytest.fail("tests/golden/fullsize.json is missing (python tests/golden/make_fullsize.py)")
    doc = json.loads(FULLSIZE.read_text())
    if key not in doc:
        pytest.fail(f"tests/golden/fullsize.json has no '{key}' row")
    return doc[key]


def _sha_len(b):
    return len(b), hashlib.sha256(b).hexdigest()


def test_chain_4gib_128_pairs_digest(cr_lib):
    """The 128-pair chain at its stated size: 4 GiB of tiled Zipf text, Session.apply_batch
    (lengths chained on the device), output digest equal to the chained bytes.replace."""
    g = _fullsize("c3")
    txt, pairs = WL.c3_input(g["generator"]["total"], seed=g["generator"]["seed"])
    assert len(txt) == g["in_len"]
    with Wr.Session(cr_lib, txt) as s:
        del txt
        n = s.apply_batch(pairs)
        out = s.result()
    assert n == g["out_len"]
    assert _sha_len(out) == (g["out_len"], g["out_sha256"])


def test_stream_16gib_8_pairs_digest(cr_lib):
    """Streaming at its stated size: 16 GiB of tiled Zipf text, a pattern planted across every
    256 MiB chunk boundary, 8 mixed pairs, through gpu_replace_streaming (chunk-major native
    path); output digest equal to the chained bytes.replace."""
    g = _fullsize("c4")
    gen = g["generator"]
    buf, pairs, planted = WL.c4_input(gen["total"], chunk=gen["chunk"], seed=gen["seed"])
    assert len(buf) == g["in_len"] and planted == g["planted"]
    out = Wr.gpu_replace_streaming(cr_lib, buf, pairs, chunk_bytes=gen["chunk"])
    del buf
    assert _sha_len(out) == (g["out_len"], g["out_sha256"])


def test_first_1000_jobs_served_digests(cr_lib):
    """The first 1000 jobs of the batched-jobs generator at full size (4 KiB-64 MiB, 1-16 pairs
    each) through the request loop; every job's output digest equal to its chained
    bytes.replace."""
    rows = _fullsize("c5")["jobs"]
    assert len(rows) == 1000
    with Wr.Server(cr_lib) as srv:
        for lo in range(0, len(rows), 100):  # 100 jobs in flight at a time (bounded host memory)
            jobs = [WL.c5_job(r["job_id"]) for r in rows[lo:lo + 100]]
            tickets = [srv.submit(j.data, j.pairs) for j in jobs]
            for j, t, r in zip(jobs, tickets, rows[lo:lo + 100]):
                out = srv.wait(t)
                assert (len(j.data), len(j.pairs)) == (r["in_len"], r["npairs"])
                assert _sha_len(out) == (r["out_len"], r["out_sha256"]), f"job {r['job_id']}"
