"""Host logic of the Python binding (cuda_replace_b200.cuda_replace_wrapper), run against a
CPU test double of the C ABI (tests/fake_capi.c). Covers the chunked streaming helper
whose arithmetic (halo, carry-in, cut points) is pure host code. CPU only."""
import random

import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr


@pytest.fixture(scope="module")
def fake(fake_lib_path):
    return Wr.CudaReplaceLib(fake_lib_path)


def test_unified_and_session_roundtrip(fake):
    assert fake.unified(b"hello world hello universe", b"hello", b"goodbye") == b"goodbye world goodbye universe"
    with Wr.Session(fake, b"aaabaaabaaa") as s:
        assert s.apply(b"aaa", b"X") == 5
        assert s.result() == b"XbXbX"
        assert s.length() == 5
        assert s.apply_batch([(b"X", b"YY"), (b"b", b"")]) == 6
        assert s.result() == b"YYYYYY"
        s.reset(b"abcabc")
        assert s.apply_seeded(b"abc", b"Z", -3) == (2, 3)
        assert s.query_prefix(4) == (2, 3)


def test_unified_large_fills_exact_bytes(fake):
    """unified() on inputs from 4 MiB writes into a bytes object of the worst-case length and
    shrinks it to the result: shrinking, expanding and unchanged lengths, and an expansion
    beyond the worst-case rule (taken by the page-locked result path instead)."""
    import sys

    src = (b"xaay" * (1 << 20)) + b"aa"
    for pat, rep in ((b"aa", b"Q"), (b"a", b"bcd"), (b"zz", b"Q"), (b"y", b"")):
        got = fake.unified(src, pat, rep)
        assert type(got) is bytes and got == src.replace(pat, rep), (pat, rep)
        assert sys.getrefcount(got) == 2  # the variable and the call's argument: nothing leaked
        assert hash(got) == hash(bytes(got))
    big = fake.unified(src, b"x", b"0123456789")  # worst case 10 n: above 4 n + 64 MiB at 16 MiB
    assert big == src.replace(b"x", b"0123456789")


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        Wr.CudaReplaceLib(str(tmp_path / "nope.so"))


def test_error_codes_raise(fake):
    with Wr.Session(fake, b"abc") as s:
        with pytest.raises(RuntimeError):
            s.apply(b"x" * 9000, b"")  # longer than CUDA_REPLACE_MAX_PATTERN -> rc -4


@pytest.mark.parametrize("chunk", [1, 2, 3, 4, 5, 7, 8, 16, 1000])
def test_streaming_straddles_match_chain(fake, chunk):
    src = b"xxxaayyy" * 3 + b"aaaaaaa" + b"abababab"
    pairs = [(b"aa", b"X"), (b"X", b"bcd"), (b"abab", b""), (b"yb", b"QQQ"), (b"", b"-")]
    assert Wr.gpu_replace_streaming(fake, src, pairs, chunk_bytes=chunk) == _chain(src, pairs)


def test_streaming_reference_defect_d3(fake):
    # the reference helper returns b"xxxayyy" here (cuda_replace_wrapper.py:356); bytes.replace gives:
    assert Wr.gpu_replace_streaming(fake, b"xxxaayyy", [(b"aa", b"X")], chunk_bytes=4) == b"xxxXyyy"


def test_streaming_random(fake):
    rng = random.Random(99)
    for _ in range(300):
        alpha = rng.choice([b"a", b"ab", b"abc"])
        src = bytes(rng.choice(alpha) for _ in range(rng.randint(0, 90)))
        pairs = []
        for _ in range(rng.randint(1, 3)):
            pat = bytes(rng.choice(alpha) for _ in range(rng.randint(1, 5)))
            rep = bytes(rng.choice(b"abXY") for _ in range(rng.randint(0, 6)))
            pairs.append((pat, rep))
        chunk = rng.randint(1, 20)
        assert Wr.gpu_replace_streaming(fake, src, pairs, chunk_bytes=chunk) == _chain(src, pairs), (src, pairs, chunk)


def test_chunk_plan_covers_input():
    assert Wr.stream_chunk_plan(10, 4) == [(0, 4), (4, 8), (8, 10)]
    assert Wr.stream_chunk_plan(0, 4) == []
    assert Wr.stream_chunk_plan(3, 0) == [(0, 1), (1, 2), (2, 3)]


def _chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src
