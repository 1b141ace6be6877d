"""apply_batch with multi-pattern stages on the GPU: runs of pairs that the planner proved
independent are applied in one pass of the sm_100a kernel (kModeMulti). Every result must equal
the chained bytes.replace (the reference's apply_batch loop, cuda_replace.cu:2480-2519), and the
number of launches must equal the number of planned passes."""
import random

import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu

MiB = 1 << 20


def chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


def batch(lib, src, pairs):
    with Wr.Session(lib, src) as s:
        _, l0 = s.stats()
        n = s.apply_batch(pairs)
        _, l1 = s.stats()
        out = s.result()
    assert n == len(out)
    return out, l1 - l0


def test_entity_chain_in_few_passes(cr_lib):
    """The 128 entity pairs on Zipf text: far fewer launches than pairs, same bytes."""
    txt = WL.text_corpus(8 * MiB + 12345, seed=3)
    pairs = WL.c3_pairs(3)
    out, launches = batch(cr_lib, txt, pairs)
    assert out == chain(txt, pairs)
    assert launches <= 17


def test_random_chains_with_runs(cr_lib):
    """Random short patterns over small alphabets (runs form often) on texts of 1 byte to 300 KiB,
    so matches fall across 64-byte segments, 2 KiB warp regions, 16 KiB sub-tiles and 64 KiB
    super-tiles; expansions up to 64 bytes per match."""
    rng = random.Random(11)
    for trial in range(160):
        alpha = rng.choice([b"ab", b"abc", b"a&;x", b"xyz01", b"ab&;cd"])
        pairs = []
        for _ in range(rng.randint(2, 12)):
            p = bytes(rng.choice(alpha) for _ in range(rng.randint(1, 6)))
            r = bytes(rng.choice(alpha + b"QRS") for _ in range(rng.choice([0, 1, 2, 3, 8, 40, 64])))
            pairs.append((p, r))
        n = rng.choice([1, 15, 63, 64, 65, 2047, 2049, 16383, 16385, 65535, 65537, 140000, 300000])
        pieces = [p for p, _ in pairs] + [r for _, r in pairs] + [bytes([c]) for c in alpha + b"z"]
        src = b"".join(rng.choice(pieces) for _ in range(n // 2 + 1))[:n]
        out, _ = batch(cr_lib, src, pairs)
        assert out == chain(src, pairs), f"trial {trial}"


def test_dense_matches_and_large_expansion(cr_lib):
    """Every byte a match (one-byte patterns), replacements up to 64 bytes: the expansion
    outgrows the warps' staging and the sub-tile is written through windows."""
    pairs = [(b"a", b"X" * 64), (b"b", b""), (b"c", b"YZ"), (b"d", b"W" * 33), (b"e", b"e")]
    rng = random.Random(3)
    for n in (1000, 70000, 600000):
        src = bytes(rng.choice(b"abcde") for _ in range(n))
        out, launches = batch(cr_lib, src, pairs)
        assert out == chain(src, pairs)
        assert launches == 2  # four pairs in one pass, the last pair alone


def test_entities_back_to_back(cr_lib):
    """Entity tokens with nothing between them, across every boundary of the kernel's tiling."""
    toks = WL.entity_tokens(3)
    pairs = WL.c3_pairs(3)
    rng = random.Random(5)
    src = b"".join(rng.choice(toks) for _ in range(200000))
    out, _ = batch(cr_lib, src, pairs)
    assert out == chain(src, pairs)
