"""Parity of libcuda_replace.so (sm_100a) with the oracle: CPython bytes.replace, chained
per pair, and the C restatement for seeded applies and prefix queries. Every call goes
through the C ABI. Bit-exact is the only acceptable result."""
import hashlib
import json
import random
from pathlib import Path

import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "vectors.json").read_text())
TILE = 16384


def sha(b):
    return hashlib.sha256(b).hexdigest()


def recipe_bytes(recipe):
    return b"".join(bytes.fromhex(u) * c for u, c in recipe)


def chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


@pytest.mark.parametrize("row", GOLDEN["known_answer"] + GOLDEN["defects"], ids=lambda r: r["name"])
def test_golden_vectors(cr_lib, row):
    src = recipe_bytes(row["recipe"])
    pairs = [(bytes.fromhex(p), bytes.fromhex(r)) for p, r in row["pairs"]]
    if len(pairs) == 1:
        out = cr_lib.unified(src, *pairs[0])
        assert len(out) == row["out_len"] and sha(out) == row["out_sha256"]
    with Wr.Session(cr_lib, src) as s:
        for p, r in pairs:
            s.apply(p, r)
        out = s.result()
    assert len(out) == row["out_len"] and sha(out) == row["out_sha256"]


@pytest.mark.parametrize("row", GOLDEN["configs"], ids=lambda r: r["name"])
def test_config_digests(cr_lib, row):
    from tests.golden.make_golden import config_inputs
    src, pairs = config_inputs(row)
    with Wr.Session(cr_lib, src) as s:
        n = s.apply_batch(pairs)
        out = s.result()
    assert n == row["out_len"] and len(out) == row["out_len"] and sha(out) == row["out_sha256"]


def test_random_small_cases(cr_lib):
    rng = random.Random(2024)
    alphabets = [b"a", b"ab", b"aab", b"abc", b"\x00\x01", bytes(range(7))]
    with Wr.Session(cr_lib, b"") as s:
        for _ in range(1500):
            alpha = rng.choice(alphabets)
            src = bytes(rng.choice(alpha) for _ in range(rng.randint(0, 70)))
            pat = bytes(rng.choice(alpha) for _ in range(rng.randint(0, 7)))
            rep = bytes(rng.choice(b"XY\x00z") for _ in range(rng.randint(0, 9)))
            s.reset(src)
            n = s.apply(pat, rep)
            out = s.result()
            assert out == src.replace(pat, rep), (src, pat, rep, out)
            assert n == len(out)


PATTERNS = [b"a", b"aa", b"aaa", b"ab", b"aba", b"abab", b"ACGT", b"a" * 5, b"a" * 31, b"a" * 32,
            b"a" * 33, b"a" * 63, b"a" * 64, b"a" * 65, b"ab" * 40, b"a" * 257, b"aab" * 100 + b"a",
            b"xyz" * 90 + b"q"]


@pytest.mark.parametrize("pat", PATTERNS, ids=lambda p: f"L{len(p)}-{p[:6]!r}")
def test_periodic_runs_across_tiles(cr_lib, pat):
    """Long runs where every position is a candidate: the carry between tiles decides
    every kept start (the reference's tile-carry defect lives here)."""
    sizes = [TILE - 1, TILE, TILE + 1, 3 * TILE + 17, 20000, 40001, 200_003]
    with Wr.Session(cr_lib, b"") as s:
        for n in sizes:
            for base in (b"a", b"ab", b"aab"):
                src = (base * (n // len(base) + 1))[:n]
                for rep in (b"", b"X", b"QRS", b"0123456789" * 3):
                    s.reset(src)
                    s.apply(pat, rep)
                    assert s.result() == src.replace(pat, rep), (n, base, pat[:8], len(pat), rep)


def test_runs_with_sparse_breaks(cr_lib):
    """Multi-MB runs broken at a few random places: most 64 KiB super-tiles are covered by
    kept matches end to end (pass B writes them from the tables alone), the broken ones and
    their neighbours are not; every carry across the breaks has to line up."""
    rng = random.Random(77)
    for base, pats in ((b"a", (b"a", b"aa", b"aaa", b"a" * 5, b"a" * 32, b"a" * 33)),
                       (b"ab", (b"ab", b"abab", b"aba", b"b"))):
        n = 3_000_017
        src = bytearray((base * (n // len(base) + 1))[:n])
        for _ in range(25):
            i = rng.randrange(n)
            src[i:i + 1] = rng.choice((b"c", b"b", b"a"))
        src = bytes(src)
        for pat in pats:
            for rep in (b"", b"X", b"QRS", b"0123456789" * 3):
                assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep), (base, pat, rep)


def test_region_blocks_copy_or_replace(cr_lib):
    """Inputs made of 2 KiB blocks (one warp region each) that are runs of the pattern's byte,
    of another byte, or random: whole super-tiles whose regions are each a copy or a run of
    replacements take the table-driven pass B, the others the general one."""
    rng = random.Random(91)
    blocks = []
    for _ in range(1500):
        k = rng.random()
        blocks.append(b"a" * 2048 if k < 0.45 else (b"b" * 2048 if k < 0.9 else rng.randbytes(2048)))
    src = b"".join(blocks) + b"aaab"
    for pat, rep in ((b"a", b"XY"), (b"a", b""), (b"aa", b"Q"), (b"aaa", b""), (b"b", b"cd"), (b"ab", b"Z"),
                     (b"aab", b"0123")):
        assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep), (pat, rep)


def test_runs_ending_near_region_edges(cr_lib):
    """Runs of one byte that end 0-4 bytes past a 2 KiB warp region, or just before one: the
    windows that start at the end of a uniform region reach into the next one."""
    rng = random.Random(17)
    parts = []
    for _ in range(600):
        k = rng.randrange(1, 4)
        parts.append(b"a" * (2048 * k + rng.choice((-3, -2, -1, 0, 1, 2, 3, 4))) + rng.choice((b"b", b"ab", b"ba", b"c")))
    src = b"".join(parts)
    for pat, rep in ((b"a", b"XY"), (b"aa", b"Q"), (b"aaa", b""), (b"aaaa", b"Z"), (b"aaaaa", b"12"),
                     (b"a" * 9, b""), (b"aab", b"R"), (b"aaab", b"")):
        assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep), (pat, rep)


def test_large_inputs_unified_and_stream(cr_lib):
    """Inputs above 256 MiB through unified() and through the native chunk-major stream with
    one pair (chunks of n/8): results equal bytes.replace, also for matches planted across every
    chunk join, with expansion (the stream sizes its result for n/L matches), deletion and a
    bordered pattern."""
    n = (256 << 20) + 12345
    chunk = max(32 << 20, ((n // 8 + (1 << 20) - 1) >> 20) << 20)
    rng = random.Random(23)
    text = bytearray(rng.randbytes(1 << 20) * (n // (1 << 20) + 1))[:n]
    for c in range(chunk, n, chunk):  # a match straddling every join
        text[c - 2:c + 3] = b"&amp;"
        text[c - 7:c - 4] = b"aab"
    text = bytes(text)
    for pat, rep in ((b"&amp;", b"&"), (b"&amp;", b"<entity>"), (b"aab", b""), (b"\x00", b"0123")):
        want = text.replace(pat, rep)
        assert cr_lib.unified(text, pat, rep) == want, (pat, rep)
        assert _native_stream(cr_lib, text, [(pat, rep)], chunk) == want, (pat, rep)
    run = b"a" * n
    for pat, rep in ((b"aa", b"X"), (b"a", b"bcd")):
        want = run.replace(pat, rep)
        assert cr_lib.unified(run, pat, rep) == want, (pat, rep)
        assert _native_stream(cr_lib, run, [(pat, rep)], chunk) == want, (pat, rep)


def test_unified_page_locked_large_chunked(cr_lib):
    """unified() on an input of 256 MiB or more takes the chunked path (uploads, replaces and
    downloads of up to sixteen chunks overlapped; a pageable input staged chunk by chunk through
    page-locked buffers by a producer thread): results equal bytes.replace, also
    for matches planted across every chunk join, for bordered and free patterns, expansion and
    deletion."""
    import ctypes as C

    import torch

    n = (300 << 20) + 777
    chunk = max(32 << 20, ((n + 15) // 16 + (1 << 20) - 1) >> 20 << 20)
    rng = random.Random(41)
    text = bytearray(rng.randbytes(1 << 20) * (n // (1 << 20) + 1))[:n]
    for j in range(chunk, n - chunk // 2, chunk):
        # a chunk's replace starts at j, its upload at j + L - 1: matches straddle both joins
        for c in (j, j + 4, j + 3, j + 1):
            text[c - 2 + 64 * (c - j):c + 3 + 64 * (c - j)] = b"&amp;"
        text[j - 3:j + 1] = b"abab"      # straddles the join by one byte
        text[j + 200:j + 204] = b"abab"
        text[j + 256 - 4:j + 256] = b"abab"
    text = bytes(text)
    run = b"a" * n
    out_ptr = C.POINTER(C.c_uint8)()
    out_len = C.c_size_t()
    for src, cases in ((text, ((b"&amp;", b"&"), (b"&amp;", b"<e>"), (b"abab", b"X"), (b"\x00", b""))),
                       (run, ((b"aa", b"X"), (b"a", b"bcd"), (b"aaa", b"")))):
        h = torch.frombuffer(bytearray(src), dtype=torch.uint8).pin_memory()
        # page-locked (every upload queued at once) and pageable (staged by a producer thread)
        for pinned, pat, rep in [(True, pt, rp) for pt, rp in cases] + [(False, pt, rp) for pt, rp in cases[:2]]:
            ptr = C.cast(h.data_ptr(), C.POINTER(C.c_uint8)) if pinned else C.cast(C.c_char_p(src), C.POINTER(C.c_uint8))
            pb, rb = C.create_string_buffer(pat, len(pat)), C.create_string_buffer(rep, len(rep) or 1)
            rc = cr_lib.lib.cuda_replace_unified(ptr, n,
                                                 C.cast(pb, C.POINTER(C.c_uint8)), len(pat),
                                                 C.cast(rb, C.POINTER(C.c_uint8)), len(rep),
                                                 C.byref(out_ptr), C.byref(out_len))
            assert rc == 0
            got = C.string_at(out_ptr, out_len.value) if out_len.value else b""
            if out_len.value:
                cr_lib.lib.cuda_free_host(out_ptr)
            assert got == src.replace(pat, rep), (pat, rep)
        del h


def test_unified_into_caller_buffer(cr_lib):
    """cuda_replace_unified_into writes the result into caller memory: the chunked path (input
    of 256 MiB or more, output downloaded in 32 MiB pieces through page-locked slots and copied
    out meanwhile) and the single-launch one (smaller inputs; results above and below one piece)
    equal bytes.replace, also for matches across the chunk joins; a buffer below the result
    length returns 1 with the length needed; CudaReplaceLib.unified takes this path for large
    inputs and returns exact bytes objects."""
    import ctypes as C

    U8P = C.POINTER(C.c_uint8)
    n = (300 << 20) + 777
    chunk = max(32 << 20, ((n + 15) // 16 + (1 << 20) - 1) >> 20 << 20)
    rng = random.Random(43)
    text = bytearray(rng.randbytes(1 << 20) * (n // (1 << 20) + 1))[:n]
    for j in range(chunk, n - chunk // 2, chunk):
        text[j - 3:j + 1] = b"abab"  # straddles the join by one byte
        text[j + 100:j + 104] = b"abab"
    text = bytes(text)
    run = b"a" * n

    def call(src, pat, rep, cap):
        dst = C.create_string_buffer(max(cap, 1))
        got = C.c_size_t()
        pb, rb = C.create_string_buffer(pat, len(pat)), C.create_string_buffer(rep, len(rep) or 1)
        rc = cr_lib.lib.cuda_replace_unified_into(C.cast(C.c_char_p(src), U8P), len(src), C.cast(pb, U8P), len(pat),
                                                   C.cast(rb, U8P), len(rep), dst, cap, C.byref(got))
        return rc, got.value, dst

    def bound(n_, pat, rep):
        b = C.c_size_t()
        assert cr_lib.lib.cuda_replace_output_bound(n_, len(pat), len(rep), C.byref(b)) == 0
        return b.value

    for src, pat, rep in ((text, b"abab", b"X"), (text, b"\x00", b""), (run, b"a", b"bcd"), (run, b"aa", b"X")):
        want = src.replace(pat, rep)
        rc, m, dst = call(src, pat, rep, bound(len(src), pat, rep))
        assert rc == 0 and m == len(want), (pat, rep, rc, m)
        assert C.string_at(dst, m) == want, (pat, rep)
        del dst
        assert cr_lib.unified(src, pat, rep) == want, (pat, rep)
    # single-launch path: a result above one 32 MiB piece, one below it, and an empty one
    for size, pat, rep in ((80 << 20, b"a", b"bc"), (5 << 20, b"aa", b"X"), (6 << 20, b"a", b"")):
        src = b"a" * size
        want = src.replace(pat, rep)
        rc, m, dst = call(src, pat, rep, bound(size, pat, rep))
        assert rc == 0 and m == len(want) and C.string_at(dst, m) == want, (size, pat, rep)
        assert cr_lib.unified(src, pat, rep) == want
    # too small a buffer: 1 and the length needed, on both paths
    for src in (run, b"a" * (8 << 20)):
        rc, m, _ = call(src, b"a", b"bcd", len(src))
        assert rc == 1 and m == 3 * len(src)
    # after the refusals, the cached session still works
    assert cr_lib.unified(b"xaay" * (2 << 20), b"aa", b"Q") == b"xQy" * (2 << 20)


def test_pieces_threshold_in_regions(cr_lib):
    """Free-mode super-tiles whose 2 KiB warp regions hold 0-64 matches: regions with at most 16
    are written as literal runs between replacements (table-driven pass B), a super-tile with a
    region above 16 takes the general pass B. Matches at region starts and ends, straddling
    region and super-tile edges, back to back, shrinking, deleting and expanding: bytes.replace
    exactly, through Session.apply (one launch) and unified."""
    rng = random.Random(47)
    pat = b"&te;"
    region, super_tile = 2048, 4 * TILE
    n = 96 * super_tile + 777
    buf = bytearray(rng.choice(b"abcdefgh ;") for _ in range(n))
    counts = [0, 1, 2, 3, 15, 16, 17, 31, 32, 64]
    for r in range(n // region - 1):
        k = counts[r % len(counts)] if (r // 32) % 3 else counts[(r * 7) % 6]  # some super-tiles stay <= 16
        base = r * region
        if k == 0:
            continue
        if r % 5 == 0:  # back to back from the region start
            pos = [base + 4 * i for i in range(k)]
        else:
            pos = sorted(rng.sample(range(base, base + region - 4, 4), k))
        for q in pos:
            buf[q:q + 4] = pat
    for e in range(super_tile, n - 8, super_tile):  # straddling super-tile edges
        off = rng.randrange(1, 4)
        buf[e - off:e - off + 4] = pat
    for e in range(region * 3, n - 8, region * 11):  # straddling region edges
        buf[e - 2:e + 2] = pat
    src = bytes(buf)
    for rep in (b"6n", b"", b"XYZ12345", b"&"):
        want = src.replace(pat, rep)
        with Wr.Session(cr_lib, src) as s:
            assert s.apply(pat, rep) == len(want)
            assert s.result() == want, rep
        assert cr_lib.unified(src, pat, rep) == want, rep


def test_fuzz_runs_blocks_and_text(cr_lib):
    """Seeded inputs of 1-3 MB mixing runs of one byte (often whole 2 KiB regions), short-alphabet
    text and random bytes, against bordered and free patterns of 1-6 bytes and replacements of
    0-8 bytes: every pass-B mode (no input, table-driven, general) and the uniform-region test
    meet each other at super-tile edges."""
    pats = [b"a", b"aa", b"aaa", b"ab", b"aba", b"b", b"ba", b"abab", b"aab", b"aaaaaa", b"\x00"]
    for seed in range(24):
        rng = random.Random(1000 + seed)
        parts, size = [], rng.randrange(1 << 20, 3 << 20)
        total = 0
        while total < size:
            k = rng.random()
            if k < 0.35:
                part = rng.choice(b"ab").to_bytes(1, "little") * rng.choice((2048, 4096, rng.randrange(1, 20000)))
            elif k < 0.7:
                part = bytes(rng.choice(b"ab") for _ in range(rng.randrange(1, 3000)))
            elif k < 0.85:
                part = bytes(rng.choice(b"abc") for _ in range(rng.randrange(1, 3000)))
            else:
                part = rng.randbytes(rng.randrange(1, 5000))
            parts.append(part)
            total += len(part)
        src = b"".join(parts)
        for _ in range(3):
            pat = rng.choice(pats)
            rep = bytes(rng.choice(b"XYZ") for _ in range(rng.randrange(0, 9)))
            assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep), (seed, pat, rep)


def test_tile_boundary_straddles(cr_lib):
    rng = random.Random(5)
    for L in (2, 3, 4, 5, 8, 16, 64, 65, 100, 300):
        pat = bytes(rng.randrange(256) for _ in range(L))
        src = bytearray(rng.randrange(256) for _ in range(5 * TILE + 77))
        for b in range(TILE, len(src) - L, TILE):
            for off in (1, L // 2, L - 1):
                s0 = b - off
                src[s0:s0 + L] = pat
        src = bytes(src)
        for rep in (b"", b"#", bytes(L + 7)):
            assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep)


def test_expansion_windows(cr_lib):
    # each 16 KiB input tile expands to ~3.2 MB of output: many output windows per tile
    src = b"a" * (3 * TILE + 5) + b"b" * 1000
    for rep in (b"x" * 200, bytes(range(256)) * 20):
        assert cr_lib.unified(src, b"a", rep) == src.replace(b"a", rep)


def test_long_patterns_and_replacements(cr_lib):
    rng = random.Random(11)
    for L, R in ((257, 3), (300, 8192), (1000, 1), (4096, 4096), (8192, 0), (8192, 8192)):
        pat = bytes(rng.randrange(256) for _ in range(L))
        rep = bytes(rng.randrange(256) for _ in range(R))
        filler = bytes(rng.randrange(256) for _ in range(3 * L + 100))
        src = filler + pat + pat + filler[:L // 2] + pat + filler
        assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep)
    # bordered long pattern over a periodic text (tile tables beyond the warp level)
    pat = b"ab" * 300
    src = b"ab" * 40000
    assert cr_lib.unified(src, pat, b"Z") == src.replace(pat, b"Z")


def test_too_long_pattern_is_rejected(cr_lib):
    with Wr.Session(cr_lib, b"abc") as s:
        with pytest.raises(RuntimeError, match="rc=-4"):
            s.apply(b"p" * 8193, b"")


def test_seeded_apply_and_query_prefix(cr_lib, oracle_mod):
    rng = random.Random(77)
    with Wr.Session(cr_lib, b"") as s:
        for trial in range(60):
            base = rng.choice([b"a", b"ab", b"aab", b"abc"])
            n = rng.choice([10, 100, TILE + 3, 3 * TILE, 70000])
            src = bytearray((base * (n // len(base) + 1))[:n])
            for _ in range(rng.randint(0, 20)):
                src[rng.randrange(n)] = ord("z")
            src = bytes(src)
            pat = (base * 8)[:rng.randint(1, 6)]
            rep = b"R" * rng.randint(0, 4)
            seed = rng.choice([-(1 << 40), -(1 << 29), -3, -2, -1, 0, 5, n // 2])
            s.reset(src)
            new_len, last = s.apply_seeded(pat, rep, seed)
            bb = oracle_mod.block_before_from_seed(seed, len(pat))
            exp, kept, exp_last = oracle_mod.replace(src, pat, rep, bb)
            assert s.result() == exp
            assert new_len == len(exp) and last == exp_last
            for lim in sorted({0, 1, n // 3, n // 2, TILE - 1, TILE, TILE + 1, n - 1, n, n + 5}):
                if lim < 0:
                    continue
                assert s.query_prefix(lim) == oracle_mod.query_prefix(src, pat, lim, bb), (trial, lim)


def test_query_prefix_int_abi(cr_lib):
    import ctypes as C
    with Wr.Session(cr_lib, b"abcabcabc") as s:
        s.apply(b"abc", b"X")
        k, l = C.c_int(0), C.c_int(0)
        assert cr_lib.lib.cuda_replace_query_prefix(s.h, 7, C.byref(k), C.byref(l)) == 0
        assert (k.value, l.value) == (3, 6)


def test_streaming_helper_with_planted_straddles(cr_lib):
    txt = WL.text_corpus(3 << 20, seed=4)
    pairs = WL.c4_pairs(seed=4)
    chunk = 256 << 10
    for pat, _ in pairs[:3]:
        txt, _count = WL.plant_across_boundaries(txt, pat, chunk, seed=len(pat))
    assert Wr.gpu_replace_streaming(cr_lib, txt, pairs, chunk_bytes=chunk) == chain(txt, pairs)


def test_c1_full_size(cr_lib):
    data, pat, rep = WL.c1_acgt()
    assert cr_lib.unified(data, pat, rep) == data.replace(pat, rep)


def test_apply_batch_empty_and_null_pairs(cr_lib):
    with Wr.Session(cr_lib, b"hello") as s:
        assert s.apply_batch([]) == 5
        assert s.apply_batch([(b"", b"-"), (b"-h", b"H")]) == 10
        assert s.result() == b"hello".replace(b"", b"-").replace(b"-h", b"H")


def test_launch_counter_counts_kernels(cr_lib):
    with Wr.Session(cr_lib, b"a" * 100000) as s:
        _, l0 = s.stats()
        s.apply(b"aa", b"b")
        s.apply(b"b", b"cc")
        kept, l1 = s.stats()
        assert l1 - l0 == 2 and kept == 50000


def test_apply_batch_chained_matches_pairwise(cr_lib, oracle_mod):
    """apply_batch chains lengths on the device (no host round trip per pair); the result,
    the final length and the following query_prefix must equal the pair-by-pair chain."""
    rng = random.Random(31)
    base = WL.text_corpus(600_000, seed=7)
    for trial in range(6):
        pairs = []
        for _ in range(rng.choice([2, 3, 7, 16])):
            w = rng.choice([b"aa", b"a", b"ab", b"the", b"e ", b"&amp;", b"xyz", b"\n", b"ss"])
            rep = bytes(rng.choice(b"QRS") for _ in range(rng.randint(0, 5)))
            pairs.append((w, rep))
        src = base[: rng.randint(1, len(base))]
        exp = src
        for p_, r_ in pairs:
            exp = exp.replace(p_, r_)
        with Wr.Session(cr_lib, src) as s:
            n = s.apply_batch(pairs)
            assert n == len(exp) and s.length() == len(exp)
            assert s.result() == exp
            # query_prefix describes the last pair applied to the second-to-last output
            prev = src
            for p_, r_ in pairs[:-1]:
                prev = prev.replace(p_, r_)
            lp = pairs[-1][0]
            for lim in (0, len(prev) // 3, len(prev)):
                assert s.query_prefix(lim) == oracle_mod.query_prefix(prev, lp, lim), (trial, lim)


def _native_stream(cr_lib, src, pairs, chunk):
    out = Wr.stream_native(cr_lib, src, pairs, chunk)
    assert out is not None, "cuda_replace_stream rejected a supported pair list"
    return out


@pytest.mark.parametrize("chunk", [1, 7, 16, 255, 4096, 16384 + 3, 1 << 20])
def test_native_stream_small_chunks(cr_lib, chunk):
    """Chunk-major streaming: every pair holds L-1 bytes back per chunk and carries match
    coverage into the next chunk; the result must equal chained bytes.replace for any cut."""
    rng = random.Random(chunk)
    for trial in range(4):
        base = rng.choice([b"a", b"ab", b"aab", b"abc"])
        n = rng.choice([n for n in (1, 50, 5000, 70000) if n <= 400 * chunk])
        src = bytearray((base * (n // len(base) + 1))[:n])
        for _ in range(rng.randint(0, 30)):
            src[rng.randrange(n)] = ord("z")
        src = bytes(src)
        pairs = []
        for _ in range(rng.randint(1, 5)):
            pat = (base * 8)[:rng.randint(1, 6)]
            rep = bytes(rng.choice(b"abzQ") for _ in range(rng.randint(0, 5)))
            pairs.append((pat, rep))
        assert _native_stream(cr_lib, src, pairs, chunk) == chain(src, pairs), (chunk, trial, pairs)


def test_native_stream_planted_straddles(cr_lib):
    txt = WL.text_corpus(6 << 20, seed=9)
    pairs = WL.c4_pairs(seed=9)
    chunk = 1 << 20
    for pat, _ in pairs[:4]:
        txt, _count = WL.plant_across_boundaries(txt, pat, chunk, seed=len(pat) + 1)
    exp = chain(txt, pairs)
    assert _native_stream(cr_lib, txt, pairs, chunk) == exp
    assert _native_stream(cr_lib, bytearray(txt), pairs, chunk) == exp
    assert Wr.gpu_replace_streaming(cr_lib, txt, pairs, chunk_bytes=chunk) == exp


def test_native_stream_expansion_regrows(cr_lib):
    # outputs far above the planned capacity: stages overflow and the chunk runs again
    src = b"a" * 3_000_000 + b"b" * 1000
    pairs = [(b"a", b"Q" * 200), (b"QQ", b"RRR"), (b"b", b"")]
    assert _native_stream(cr_lib, src, pairs, 1 << 20) == chain(src, pairs)


def test_native_stream_limits_and_mixed_pairs(cr_lib):
    assert Wr.stream_native(cr_lib, b"abc", [(b"", b"x")], 16) is None
    assert Wr.stream_native(cr_lib, b"abc", [(b"ab" * 20, b"x")], 16) is None  # bordered, L > 32
    assert Wr.stream_native(cr_lib, b"abc", [(b"a" * 300, b"x")], 16) is None
    assert Wr.stream_native(cr_lib, b"", [(b"a", b"x")], 16) == b""
    assert Wr.stream_native(cr_lib, b"abc", [], 16) == b"abc"
    src = (b"ab" * 30000 + b"c") * 3
    pairs = [(b"c", b"cc"), (b"ab" * 20, b"Z"), (b"", b"-"), (b"-Z", b"z"), (b"b-", b"")]
    assert Wr.gpu_replace_streaming(cr_lib, src, pairs, chunk_bytes=10000) == chain(src, pairs)


@pytest.mark.parametrize("L,R", [(40, 40), (100, 100), (33, 64), (2048, 2048), (3000, 900), (200, 600)])
def test_matches_overhanging_warp_regions(cr_lib, L, R):
    """A match that starts near the end of a 2 KiB warp region and runs past it makes that
    region's output up to 2047 + R bytes: more than the input it covers. Plant such matches
    at every region end (and inside) and compare with bytes.replace."""
    rng = random.Random(L * 7 + R)
    pat = bytes(rng.randrange(1, 256) for _ in range(L))
    rep = bytes(rng.randrange(256) for _ in range(R))
    n = 40 * 2048 + 123
    src = bytearray(rng.randrange(256) for _ in range(n))
    pos = 2047
    while pos + L <= n:
        src[pos:pos + L] = pat
        pos += max(L + rng.randrange(0, 64), 2048 * (1 + L // 2048))
    for pos in range(5, n - L, 8192 + 1000):
        if all(src[pos + k] != 0x00 for k in range(1)):
            src[pos:pos + L] = pat
    src = bytes(src)
    assert cr_lib.unified(src, pat, rep) == src.replace(pat, rep)
