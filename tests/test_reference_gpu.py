"""Bit-exact parity of libcuda_replace.so with the reference's own GPU library, both driven
through the reference's UNCHANGED ctypes wrapper.

The reference library is cuda_replace.cu (RAZZULLIX/cuda_replace) built for sm_100a by
oracle/build_ref.py into oracle/_ref/libcuda_replace_ref.so; the same recipe copies the
reference's cuda_replace_wrapper.py beside it, byte for byte. Every call in this file goes
through that copied wrapper (CudaReplaceLib.unified py:124-141, Session py:145-297,
gpu_replace_streaming py:305-366), once with each library, so this file is also the proof that
the new library is a drop-in for the reference's binding. The reference's own check is
equality with bytes.replace (test/test.py:150-161); here the two libraries must also equal
each other byte for byte.

The reference runs only inside its envelope: input, kept count and every output below 2**31
(cuda_replace.cu truncates positions and counts to int beyond that: cu:159-160, 609, 668,
1418), on its default fused path (CUDA_REPLACE_FUSED unset, cu:2272), and never with a
pattern whose last byte is 0x00 on an expanding pair (its zero-filled halo, cu:766 and 839,
then marks a match that ends past the buffer, and the expansion scatter, cu:1561-1608, writes
past the output length it computed).

Recorded divergences, where the new library follows bytes.replace and the reference does not:
  D1  tile-carry composition in the fused path (cu:737-884): runs of a self-overlapping
      pattern longer than a tile;
  D2  zero-filled halo (cu:766): a pattern ending in 0x00 matches past the end;
  D3  the streaming helper cuts a chunk's output before the replacement of a match that
      straddles the chunk boundary (py:356): a wrapper defect, so the unchanged helper gives a
      wrong result with either library; the corrected helper of this package does not;
  D5  empty pattern: the reference returns the input unchanged (cu:2104-2109).
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
from pathlib import Path

import pytest

from cuda_replace_b200 import build as B
from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parent.parent
REF_DIR = REPO / "oracle" / "_ref"
REF_LIB = REF_DIR / "libcuda_replace_ref.so"
REF_WRAPPER = REF_DIR / "cuda_replace_wrapper.py"
GOLDEN = json.loads((Path(__file__).parent / "golden" / "vectors.json").read_text())
MiB = 1 << 20
ENVELOPE = (1 << 31) - 1


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def recipe_bytes(recipe):
    return b"".join(bytes.fromhex(u) * c for u, c in recipe)


def chain(src: bytes, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


@pytest.fixture(scope="module")
def refw():
    """The reference's wrapper module, imported from its verbatim copy."""
    if not (REF_LIB.exists() and REF_WRAPPER.exists()):
        pytest.skip("reference library not built here (oracle/build_ref.py needs the reference source)")
    os.environ.pop("CUDA_REPLACE_FUSED", None)  # the reference's default fused path (cu:2272)
    spec = importlib.util.spec_from_file_location("reference_cuda_replace_wrapper", REF_WRAPPER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def libs(refw):
    """(new, reference): both libraries bound by the reference's unchanged CudaReplaceLib."""
    if not B.LIB_PATH.exists():
        B.build()
    return refw.CudaReplaceLib(str(B.LIB_PATH)), refw.CudaReplaceLib(str(REF_LIB))


def both_unified(libs, src, pat, rep):
    return [lib.unified(src, pat, rep) for lib in libs]


def both_session_batch(refw, libs, src, pairs):
    outs = []
    for lib in libs:
        with refw.Session(lib, src) as s:
            n = s.apply_batch(pairs)
            out = s.result()
            assert n == len(out) == s.length()
        outs.append(out)
    return outs


# ------------------------------------------------------------------ the reference's own cases
@pytest.mark.parametrize("row", GOLDEN["known_answer"], ids=lambda r: r["name"])
def test_known_answers_match_reference(refw, libs, row):
    """README example, wrapper self-test and the six test.py cases (test/test.py:44-99):
    unified() and Session.apply through the reference wrapper, both libraries."""
    src = recipe_bytes(row["recipe"])
    pairs = [(bytes.fromhex(p), bytes.fromhex(r)) for p, r in row["pairs"]]
    assert len(pairs) == 1
    new, ref = both_unified(libs, src, *pairs[0])
    assert sha(new) == row["out_sha256"] and len(new) == row["out_len"]
    assert new == ref
    outs = []
    for lib in libs:
        with refw.Session(lib, src) as s:
            s.apply(*pairs[0])
            outs.append(s.result())
    assert outs[0] == outs[1] == new


def test_c1_acgt_16mib_matches_reference(libs):
    src, pat, rep = WL.c1_acgt(16 * MiB, seed=1)
    new, ref = both_unified(libs, src, pat, rep)
    assert new == ref == src.replace(pat, rep)


@pytest.mark.parametrize("case", ["aa->X", "a->bcd", "random 00 00 01->''"])
def test_c2_shapes_256mib_match_reference(libs, case):
    """The single-pair shapes of the 2 GiB / 1 GiB workload at 256 MiB (inside the
    reference's 2**31 envelope: 2**27 kept, a 768 MiB expansion, embedded NULs)."""
    n = 256 * MiB
    if case == "aa->X":
        src, pat, rep = b"a" * n, b"aa", b"X"
    elif case == "a->bcd":
        src, pat, rep = b"a" * n, b"a", b"bcd"
    else:
        import numpy as np
        src = np.random.default_rng(2).integers(0, 256, size=n, dtype=np.uint8).tobytes()
        pat, rep = b"\x00\x00\x01", b""
    new, ref = both_unified(libs, src, pat, rep)
    want = src.replace(pat, rep)
    assert len(new) == len(want) and new == want
    assert ref == new


def test_c3_text_128_pairs_64mib_matches_reference(refw, libs):
    """Session.apply_batch of the 128 entity pairs on 64 MiB of the Zipf text."""
    src = WL.text_corpus(64 * MiB, seed=3)
    pairs = WL.c3_pairs(3)
    new, ref = both_session_batch(refw, libs, src, pairs)
    assert new == chain(src, pairs)
    assert ref == new


def _c5_jobs_for_reference(count: int):
    """The first `count` jobs of the batched-jobs generator with no 0x00 byte in the input or
    in any pattern (so the reference's zero-filled halo cannot match) and whose chain stays
    inside the reference's envelope (every length at most 256 MiB)."""
    jobs, job_id = [], 0
    while len(jobs) < count:
        job = WL.c5_job(job_id)
        job_id += 1
        if b"\x00" in job.data or any(b"\x00" in p for p, _ in job.pairs):
            continue
        out, ok = job.data, True
        for p, r in job.pairs:
            out = out.replace(p, r)
            if len(out) > 256 * MiB:
                ok = False
                break
        if ok:
            jobs.append((job, out))
    return jobs, job_id


def test_c5_jobs_match_reference(refw, libs):
    """200 independent jobs (sizes log-uniform 4 KiB-64 MiB, 1-16 pairs each, pattern 1-32 B,
    replacement 0-64 B), each a Session.apply_batch through both libraries."""
    jobs, scanned = _c5_jobs_for_reference(200)
    assert len(jobs) == 200 and scanned < 2000
    for job, want in jobs:
        new, ref = both_session_batch(refw, libs, job.data, job.pairs)
        assert new == want, f"job {job.job_id}: new library differs from bytes.replace"
        assert ref == new, f"job {job.job_id}: reference differs from the new library"


# ------------------------------------------------------------------ seeded applies and queries
SEEDED = [
    ("a-run aa->X", b"a" * 8000, b"aa", b"X"),
    ("abab->Z", b"abababab" * 750 + b"ab", b"abab", b"Z"),
    ("lo->LOL", b"hello world " * 600, b"lo", b"LOL"),
    ("aa->''", b"xxxaayyy" * 1000, b"aa", b""),
]
SEEDS = (-(1 << 29), 0, 1, 5, 101)


@pytest.mark.parametrize("name,src,pat,rep", SEEDED, ids=[c[0] for c in SEEDED])
def test_seeded_apply_and_query_prefix_match_reference(refw, libs, oracle_mod, name, src, pat, rep):
    """apply_seeded with the unseeded sentinel (py:313) and with non-negative seeds, then
    query_prefix at limits across the buffer (the calls streaming makes, py:347-355): the new
    library equals the C oracle, and the reference equals the new library. Inputs stay within
    one of the reference's 8 KiB fused tiles (FUSED_TILE_BYTES, cu:79), where its seeded greedy
    is exact; out_last_rel is not compared (the reference's fused path leaves it stale,
    cu:929-934)."""
    limits = (0, 1, 2, 3, 17, 4095, 4096, 4097, len(src) // 2, len(src))
    for seed in SEEDS:
        bb = oracle_mod.block_before_from_seed(None if seed <= -(1 << 28) else seed, len(pat))
        want_out, _, _ = oracle_mod.replace(src, pat, rep, bb)
        want_q = [oracle_mod.query_prefix(src, pat, lim, bb) for lim in limits]
        answers = []
        for lib in libs:
            with refw.Session(lib, src) as s:
                new_len, _ = s.apply_seeded(pat, rep, seed)
                qs = [s.query_prefix(lim) for lim in limits]
                answers.append((new_len, qs, s.result()))
        assert answers[0] == (len(want_out), want_q, want_out), f"seed {seed}"
        assert answers[1] == answers[0], f"seed {seed}"


def test_d1_seeded_tile_carry_reference_differs(refw, libs, oracle_mod):
    """A seeded apply over a self-overlapping run longer than the reference's 8 KiB fused tile:
    an odd seed shifts the greedy's parity in tile 0, but the reference seeds tile 1 from
    tile 0's unseeded pass (cu:737-884), so its output differs (D1). The new library equals
    the oracle."""
    src, pat, rep, seed = b"a" * 10000, b"aa", b"X", 1
    want, _, _ = oracle_mod.replace(src, pat, rep, oracle_mod.block_before_from_seed(seed, 2))
    outs = []
    for lib in libs:
        with refw.Session(lib, src) as s:
            s.apply_seeded(pat, rep, seed)
            outs.append(s.result())
    assert outs[0] == want
    assert outs[1] != want


# ------------------------------------------------------------------ streaming helper
def _straddles(src: bytes, pairs, chunk: int) -> int:
    """Kept matches, over all passes of the pair-major helper, that straddle one of its chunk
    boundaries (multiples of chunk in each pass's input)."""
    from oracle import oracle as O
    count, cur = 0, src
    for p, r in pairs:
        for s in O.kept_positions(cur, p):
            if (s // chunk) != ((s + len(p) - 1) // chunk):
                count += 1
        cur = cur.replace(p, r)
    return count


def test_streaming_helper_matches_reference_without_straddles(refw, libs):
    """The reference's own gpu_replace_streaming (pair-major, py:305-366) over 4 MiB of text
    and 8 mixed shrink/expand pairs, at a chunk size where no kept match straddles a chunk
    boundary: both libraries give the chained bytes.replace."""
    src = WL.text_corpus(4 * MiB, seed=4)
    pairs = WL.c4_pairs(4)
    for chunk in (MiB + 7, MiB + 13, MiB + 101, MiB + 211, 3 * MiB // 2 + 5):
        if _straddles(src, pairs, chunk) == 0:
            break
    else:
        pytest.fail("no straddle-free chunk size found")
    want = chain(src, pairs)
    new = refw.gpu_replace_streaming(libs[0], src, pairs, chunk_bytes=chunk)
    ref = refw.gpu_replace_streaming(libs[1], src, pairs, chunk_bytes=chunk)
    assert new == want and ref == want


# ------------------------------------------------------------------ recorded divergences
def test_d1_tile_carry_reference_differs(libs):
    src, pat, rep = b"a" * 20000, b"aaa", b"X"
    new, ref = both_unified(libs, src, pat, rep)
    want = src.replace(pat, rep)
    assert new == want
    assert ref != want  # D1: the fused pass seeds each tile from unseeded predecessors


def test_d2_zero_halo_reference_differs(libs):
    src, pat, rep = b"xyz\xee", b"\xee\x00", b"Q"  # shrink: the reference's writes stay in range
    new, ref = both_unified(libs, src, pat, rep)
    assert new == src.replace(pat, rep) == src
    assert ref != src  # D2: the zero-filled halo matches past the end; the byte is dropped or garbled


def test_d3_streaming_cut_is_a_wrapper_defect(refw, libs):
    src, pairs = b"xxxaayyy", [(b"aa", b"X")]
    want = chain(src, pairs)
    assert refw.gpu_replace_streaming(libs[1], src, pairs, chunk_bytes=4) != want
    assert refw.gpu_replace_streaming(libs[0], src, pairs, chunk_bytes=4) != want
    own = Wr.CudaReplaceLib(str(B.LIB_PATH))
    assert Wr.gpu_replace_streaming(own, src, pairs, chunk_bytes=4) == want
    # straddles at every boundary of a larger input, through the corrected helper
    text = WL.text_corpus(2 * MiB, seed=4)
    for p, _ in WL.c4_pairs(4)[:2]:
        text, _ = WL.plant_across_boundaries(text, p, 64 * 1024, seed=9)
    pairs = WL.c4_pairs(4)
    assert _straddles(text, pairs, 64 * 1024) > 0
    assert Wr.gpu_replace_streaming(own, text, pairs, chunk_bytes=64 * 1024) == chain(text, pairs)


def test_d5_empty_pattern_reference_differs(libs):
    new, ref = both_unified(libs, b"abc", b"", b"-")
    assert new == b"abc".replace(b"", b"-") == b"-a-b-c-"
    assert ref == b"abc"  # D5: the reference leaves the buffer unchanged
