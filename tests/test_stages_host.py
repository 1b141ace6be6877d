"""The stage planner of apply_batch (cuda_replace_plan_stages, host code: no GPU needed).

apply_batch runs a run of consecutive pairs in one pass when the planner has proved that
applying them one after the other (the reference's loop, cuda_replace.cu:2480-2519) gives the
same bytes as replacing every occurrence of every pattern of the run at once. These tests check
the planner's decisions against that definition on random chains: for every run it forms, the
one-pass result of a pure-Python model equals the chained bytes.replace on random texts built
to contain the patterns, the replacements and their borders."""
import ctypes as C
import random

import pytest

from cuda_replace_b200 import build as B
from cuda_replace_b200 import workloads as WL


@pytest.fixture(scope="module")
def plan():
    if not B.LIB_PATH.exists():
        B.build()
    lib = C.CDLL(str(B.LIB_PATH))
    fn = lib.cuda_replace_plan_stages
    u8p = C.POINTER(C.c_uint8)
    fn.argtypes = [C.POINTER(u8p), C.POINTER(C.c_int), C.POINTER(u8p), C.POINTER(C.c_int), C.c_int, C.c_int,
                   C.POINTER(C.c_int)]
    fn.restype = C.c_int

    def run(pairs, keep_last_alone=False):
        n = len(pairs)
        keep = [C.create_string_buffer(p, len(p) + 1) for p, _ in pairs] + \
               [C.create_string_buffer(r, len(r) + 1) for _, r in pairs]
        pp = (u8p * max(n, 1))(*[C.cast(keep[i], u8p) for i in range(n)])
        rp = (u8p * max(n, 1))(*[C.cast(keep[n + i], u8p) for i in range(n)])
        pl = (C.c_int * max(n, 1))(*[len(p) for p, _ in pairs])
        rl = (C.c_int * max(n, 1))(*[len(r) for _, r in pairs])
        st = (C.c_int * max(n, 1))()
        k = fn(pp, pl, rp, rl, n, int(keep_last_alone), st)
        assert k >= 0
        return k, list(st[:n])
    return run


def chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


def one_pass(src, pairs):
    """Every occurrence of every pattern of the run, replaced at once, left to right."""
    out, i, n = bytearray(), 0, len(src)
    while i < n:
        for p, r in pairs:
            if src.startswith(p, i):
                out += r
                i += len(p)
                break
        else:
            out.append(src[i])
            i += 1
    return bytes(out)


def runs_of(pairs, stage_of):
    runs = {}
    for pr, s in zip(pairs, stage_of):
        runs.setdefault(s, []).append(pr)
    return [runs[s] for s in sorted(runs)]


def texts_for(run, rng, count=24):
    """Random texts made of the run's patterns, replacements, their pieces and stray bytes."""
    pieces = []
    for p, r in run:
        pieces += [p, r, p[:1], p[-1:], p[1:], p[:-1]]
    alphabet = sorted(set(b"".join(pieces)) | {ord("z")})
    out = []
    for _ in range(count):
        parts = []
        for _ in range(rng.randint(1, 40)):
            if rng.random() < 0.6:
                parts.append(rng.choice(pieces))
            else:
                parts.append(bytes([rng.choice(alphabet)]))
        out.append(b"".join(parts))
    return out


def test_planned_runs_equal_the_chain_on_random_pairs(plan):
    rng = random.Random(7)
    formed = 0
    for trial in range(400):
        alpha = rng.choice([b"ab", b"abc", b"a&;x", b"xyz01", b"ab&;cd"])
        pairs = []
        for _ in range(rng.randint(2, 10)):
            p = bytes(rng.choice(alpha) for _ in range(rng.randint(1, 5)))
            r = bytes(rng.choice(alpha + b"QR") for _ in range(rng.randint(0, 4)))
            pairs.append((p, r))
        k, stage_of = plan(pairs)
        assert stage_of == sorted(stage_of) and k == len(set(stage_of))
        for run in runs_of(pairs, stage_of):
            if len(run) < 2:
                continue
            formed += 1
            for t in texts_for(run, rng):
                assert one_pass(t, run) == chain(t, run), (run, t)
    assert formed > 50  # the random chains do form runs


@pytest.mark.parametrize("pairs,apart", [
    ([(b"ab", b"c"), (b"cd", b"X")], True),          # "c" + "d" forms the later pattern
    ([(b"ab", b""), (b"xy", b"Q")], True),           # an empty replacement joins x and y
    ([(b"ab", b""), (b"y", b"Q")], False),           # ...which a one-byte pattern cannot straddle
    ([(b"abc", b"1"), (b"cde", b"2")], True),        # the patterns overlap ("abcde")
    ([(b"abc", b"1"), (b"b", b"2")], True),          # one inside the other
    ([(b"aa", b"1"), (b"b", b"2")], True),           # "aa" has a border: never in a run
    ([(b"ab", b"1"), (b"ab", b"2")], True),          # the same pattern twice
    ([(b"&amp;", b"&"), (b"&lt;", b"<")], True),     # "&" + "lt;" forms the later pattern
    ([(b"&lt;", b"<"), (b"&gt;", b">"), (b"&amp;", b"&")], False),  # decoding order that is safe
])
def test_planner_keeps_interacting_pairs_apart(plan, pairs, apart):
    k, stage_of = plan(pairs)
    assert (len(set(stage_of)) == len(pairs)) == apart
    if not apart:
        t = b"a&lt;b&gt;c&amp;lt;d&amp;&amp;gt;" if pairs[0][0].startswith(b"&") else b"abyabyxy"
        assert one_pass(t, pairs) == chain(t, pairs)


def test_entity_chain_runs(plan):
    """The 128 entity pairs of the chain workload form few runs; the last pair runs alone when
    asked (apply_batch asks)."""
    pairs = WL.c3_pairs(3)
    k, stage_of = plan(pairs)
    assert k <= 16
    k2, st2 = plan(pairs, keep_last_alone=True)
    assert st2[-1] != st2[-2] and k2 in (k, k + 1)
    text = WL.text_corpus(1 << 16, seed=3)
    out = text
    for run in runs_of(pairs, stage_of):
        out = one_pass(out, run) if len(run) > 1 else out.replace(*run[0])
    assert out == chain(text, pairs)
