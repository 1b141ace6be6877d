"""Pins the oracle (CPU restatement of the reference algorithm) to the golden vectors and to
CPython bytes.replace. CPU only."""
import hashlib
import json
import random
from pathlib import Path

import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "vectors.json").read_text())


def sha(b):
    return hashlib.sha256(b).hexdigest()


def recipe_bytes(recipe):
    return b"".join(bytes.fromhex(u) * c for u, c in recipe)


def pairs_of(row):
    return [(bytes.fromhex(p), bytes.fromhex(r)) for p, r in row["pairs"]]


@pytest.mark.parametrize("row", GOLDEN["known_answer"] + GOLDEN["defects"], ids=lambda r: r["name"])
def test_known_answer_vectors(oracle_mod, row):
    src = recipe_bytes(row["recipe"])
    assert len(src) == row["in_len"]
    out = src
    for pat, rep in pairs_of(row):
        c_out, _, _ = oracle_mod.replace(out, pat, rep)
        assert c_out == out.replace(pat, rep)
        out = c_out
    assert len(out) == row["out_len"]
    assert sha(out) == row["out_sha256"]
    if "out_hex" in row:
        assert out.hex() == row["out_hex"]


def test_readme_example_literal(oracle_mod):
    # README.md:40-42 states the expected string literally
    out, kept, last = oracle_mod.replace(b"hello world hello universe", b"hello", b"goodbye")
    assert out == b"goodbye world goodbye universe" and kept == 2 and last == 12


@pytest.mark.parametrize("row", GOLDEN["seeded"], ids=lambda r: f"{r['src_hex']}-{r['prev_last_rel']}")
def test_seeded_vectors(oracle_mod, row):
    src, pat, rep = (bytes.fromhex(row[k]) for k in ("src_hex", "pat_hex", "rep_hex"))
    bb = oracle_mod.block_before_from_seed(row["prev_last_rel"], len(pat))
    out, kept, last = oracle_mod.replace(src, pat, rep, bb)
    assert out.hex() == row["out_hex"] and kept == row["kept"] and last == row["last"]
    assert oracle_mod.py_replace(src, pat, rep, bb) == out
    for lim, k, l in row["queries"]:
        assert oracle_mod.query_prefix(src, pat, lim, bb) == (k, l)


@pytest.mark.parametrize("row", GOLDEN["configs"], ids=lambda r: r["name"])
def test_config_digests(oracle_mod, row):
    from tests.golden.make_golden import config_inputs
    src, pairs = config_inputs(row)
    assert len(src) == row["in_len"] and sha(src) == row["in_sha256"]
    out = src
    for pat, rep in pairs:
        out, _, _ = oracle_mod.replace(out, pat, rep)
    assert len(out) == row["out_len"] and sha(out) == row["out_sha256"]


def test_random_small_cases_match_bytes_replace(oracle_mod):
    rng = random.Random(1234)
    alphabets = [b"a", b"ab", b"aab", b"abc", b"\x00\x01", bytes(range(5))]
    for _ in range(4000):
        alpha = rng.choice(alphabets)
        src = bytes(rng.choice(alpha) for _ in range(rng.randint(0, 60)))
        pat = bytes(rng.choice(alpha) for _ in range(rng.randint(0, 6)))
        rep = bytes(rng.choice(b"XY\x00") for _ in range(rng.randint(0, 7)))
        expect = src.replace(pat, rep)
        assert oracle_mod.replace(src, pat, rep)[0] == expect
        assert oracle_mod.py_replace(src, pat, rep) == expect
        if pat:
            n, kept, _ = oracle_mod.replace_len(src, pat, len(rep))
            assert n == len(expect) and kept == src.count(pat)


def test_seed_blocks_only_candidates(oracle_mod):
    # prev_last_rel = -1 with L = 2 blocks position 0 only; the covered byte is still emitted
    src = b"aaaaa"
    out, kept, last = oracle_mod.replace(src, b"aa", b"X", oracle_mod.block_before_from_seed(-1, 2))
    assert out == b"aXX" and kept == 2 and last == 3


def test_query_prefix_matches_kept_positions(oracle_mod):
    rng = random.Random(7)
    for _ in range(300):
        src = bytes(rng.choice(b"ab") for _ in range(rng.randint(1, 80)))
        pat = bytes(rng.choice(b"ab") for _ in range(rng.randint(1, 4)))
        bb = rng.randint(0, 5)
        kept = oracle_mod.kept_positions(src, pat, bb)
        for lim in range(len(src) + 2):
            before = [p for p in kept if p < lim]
            assert oracle_mod.query_prefix(src, pat, lim, bb) == (len(before), before[-1] if before else -1)
