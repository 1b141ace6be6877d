"""Seeded synthetic inputs with the shapes of the five benchmark configurations.

No dataset is involved: every input is generated from a seed with numpy, so a run on any
machine reproduces the same bytes.

  C1  16 MiB i.i.d. uniform over b"ACGT", pattern b"ACGT" -> b"N"
  C2  2 GiB of b"a": (i) b"aa" -> b"X", (ii) b"a" -> b"bcd"; and 1 GiB i.i.d. uniform
      bytes with b"\\x00\\x00\\x01" -> b""
  C3  Zipf(1.1) text over a 50k-word vocabulary with HTML-entity-like tokens, 128 pairs
  C4  C3-style text, 8 mixed shrink/expand pairs, matches planted across chunk boundaries
  C5  independent jobs of log-uniform size with per-job alphabets and 1-16 pairs
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

MiB = 1 << 20
GiB = 1 << 30

Pair = Tuple[bytes, bytes]


# ------------------------------------------------------------------ C1
def c1_acgt(n: int = 16 * MiB, seed: int = 1) -> Tuple[bytes, bytes, bytes]:
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, 4, size=n, dtype=np.uint8)
    data = np.frombuffer(b"ACGT", dtype=np.uint8)[idx].tobytes()
    return data, b"ACGT", b"N"


# ------------------------------------------------------------------ C2
def c2_cases(n_run: int = 2 * GiB, n_rand: int = 1 * GiB, seed: int = 2):
    """The three single-pair cases of C2 as (name, generator, pattern, replacement).

    Generators are callables so large inputs are only materialised when needed.
    """
    def run_a() -> bytes:
        return b"a" * n_run

    def rand_bytes() -> bytes:
        return np.random.default_rng(seed).integers(0, 256, size=n_rand, dtype=np.uint8).tobytes()

    return [
        ("a-run aa->X", run_a, b"aa", b"X"),
        ("a-run a->bcd", run_a, b"a", b"bcd"),
        ("random \\x00\\x00\\x01->''", rand_bytes, b"\x00\x00\x01", b""),
    ]


# ------------------------------------------------------------------ C3 / C4 text
@dataclass
class TextSpec:
    vocab_size: int = 50_000
    zipf_s: float = 1.1
    line_every: int = 80
    entity_every: int = 200
    n_entities: int = 128


def _vocab(rng: np.random.Generator, size: int) -> List[bytes]:
    lens = rng.integers(1, 13, size=size)
    letters = rng.integers(ord("a"), ord("z") + 1, size=int(lens.sum()), dtype=np.uint8).tobytes()
    out, o = [], 0
    for ln in lens:
        out.append(letters[o:o + ln])
        o += ln
    return out


def entity_tokens(seed: int = 3, count: int = 128) -> List[bytes]:
    """'&' + 2-8 lowercase letters + ';', distinct."""
    rng = np.random.default_rng(seed + 1000)
    toks, seen = [], set()
    while len(toks) < count:
        k = int(rng.integers(2, 9))
        body = rng.integers(ord("a"), ord("z") + 1, size=k, dtype=np.uint8).tobytes()
        t = b"&" + body + b";"
        if t not in seen:
            seen.add(t)
            toks.append(t)
    return toks


def text_corpus(n: int, seed: int = 3, spec: TextSpec = TextSpec()) -> bytes:
    """Zipf-distributed words joined by spaces, a newline at the first word boundary after
    every ~80 bytes, and one entity token per ~200 bytes (replacing the word there); exactly
    n bytes long. Vectorised with numpy, built in blocks of about 16 MiB."""
    rng = np.random.default_rng(seed)
    vocab = _vocab(rng, spec.vocab_size)
    toks = entity_tokens(seed, spec.n_entities)
    words = vocab + toks  # ids >= vocab_size are entity tokens
    flat = np.frombuffer(b"".join(words), dtype=np.uint8)
    wlen = np.array([len(w) for w in words], dtype=np.int64)
    wstart = np.concatenate([[0], np.cumsum(wlen)[:-1]])
    ranks = np.arange(1, spec.vocab_size + 1, dtype=np.float64)
    probs = ranks ** (-spec.zipf_s)
    probs /= probs.sum()
    cdf = np.cumsum(probs)
    out = np.empty(n, dtype=np.uint8)
    filled = 0
    mean_word = float((wlen[:spec.vocab_size] * probs).sum()) + 1.0
    while filled < n:
        m = int(min(n - filled, 16 << 20) / mean_word) + 64
        ids = np.minimum(np.searchsorted(cdf, rng.random(m)), spec.vocab_size - 1)
        off = np.cumsum(wlen[ids] + 1)
        # entity token at the first word starting after each gap of 100-300 bytes
        gaps = rng.integers(spec.entity_every // 2, spec.entity_every * 3 // 2 + 1,
                            size=int(off[-1]) // (spec.entity_every // 2) + 2)
        marks = np.cumsum(gaps)
        ent = np.unique(np.searchsorted(off, marks[marks < off[-1]]))
        ids[ent] = spec.vocab_size + rng.integers(0, spec.n_entities, size=ent.size)
        lens = wlen[ids] + 1
        off = np.cumsum(lens)
        total = int(off[-1])
        starts = off - lens
        seps = np.where(np.diff(off // spec.line_every, prepend=0) > 0, ord("\n"), ord(" ")).astype(np.uint8)
        which = np.repeat(np.arange(m), lens)
        within = np.arange(total) - starts[which]
        is_sep = within == wlen[ids][which]
        src_idx = wstart[ids][which] + np.minimum(within, wlen[ids][which] - 1)
        block = np.where(is_sep, seps[which], flat[src_idx])
        take = min(total, n - filled)
        out[filled:filled + take] = block[:take]
        filled += take
    return out.tobytes()


def c3_pairs(seed: int = 3) -> List[Pair]:
    """128 pairs mapping each entity token (4-10 B) to a 1-2 B replacement, in order."""
    rng = np.random.default_rng(seed + 2000)
    toks = entity_tokens(seed)
    pairs = []
    for t in toks:
        k = int(rng.integers(1, 3))
        rep = rng.integers(33, 127, size=k, dtype=np.uint8).tobytes()
        pairs.append((t, rep))
    return pairs


def c4_pairs(seed: int = 4) -> List[Pair]:
    """8 pairs, pattern 2-16 B taken from the text vocabulary, replacement 0-32 B."""
    rng = np.random.default_rng(seed)
    vocab = _vocab(np.random.default_rng(3), 50_000)
    pairs = []
    while len(pairs) < 8:
        w = vocab[int(rng.integers(0, 2000))]
        if not (2 <= len(w) + 1 <= 16):
            continue
        pat = w + b" "
        k = int(rng.integers(0, 33))
        rep = rng.integers(ord("A"), ord("Z") + 1, size=k, dtype=np.uint8).tobytes()
        pairs.append((pat, rep))
    return pairs


def tiled_text(total: int, seed: int, block: int = 256 * MiB) -> bytes:
    """total bytes of the Zipf text: a generated block of `block` bytes (256 MiB, twice the
    L2 cache) repeated and cut to length. This is the full-size input of the 128-pair chain
    (4 GiB) and of the streaming workload (16 GiB): generating gigabytes of Zipf text directly
    takes minutes."""
    base = text_corpus(min(total, block), seed=seed)
    if total <= len(base):
        return base[:total]
    k, rem = divmod(total, len(base))
    return b"".join([base] * k + [base[:rem]])


def c3_input(total: int = 4 * GiB, seed: int = 3) -> Tuple[bytes, List[Pair]]:
    """The 128-pair chain workload: tiled Zipf text with entity tokens and the 128 pairs."""
    return tiled_text(total, seed), c3_pairs(seed)


def c4_input(total: int = 16 * GiB, chunk: int = 256 * MiB, seed: int = 4):
    """The streaming workload: tiled Zipf text, the 8 mixed pairs, and at every multiple of
    `chunk` the pattern of pair (j mod 8) written across boundary j (1 to L-1 of its bytes
    before it), so every pair meets a match straddling a chunk boundary. Returns (bytearray,
    pairs, planted); the buffer is planted in place (no copy of the whole input)."""
    pairs = c4_pairs(seed)
    base = text_corpus(min(total, 256 * MiB), seed=seed)
    buf = bytearray(total)
    view = memoryview(base)
    for o in range(0, total, len(base)):
        m = min(len(base), total - o)
        buf[o:o + m] = view[:m]
    rng = np.random.default_rng(seed + 7)
    planted = 0
    for j, b in enumerate(range(chunk, len(buf), chunk)):
        pat = pairs[j % len(pairs)][0]
        L = len(pat)
        off = int(rng.integers(1, L))
        s = b - off
        if s < 0 or s + L > len(buf):
            continue
        buf[s:s + L] = pat
        planted += 1
    return buf, pairs, planted


def plant_across_boundaries(data: bytes, pat: bytes, chunk: int, seed: int = 4) -> Tuple[bytes, int]:
    """Overwrite bytes so that pat occurs straddling every multiple of chunk. Returns (data, count)."""
    rng = np.random.default_rng(seed)
    buf = bytearray(data)
    L = len(pat)
    count = 0
    if L < 2:
        return bytes(buf), 0
    for b in range(chunk, len(buf) - L, chunk):
        off = int(rng.integers(1, L))  # 1..L-1 bytes before the boundary
        s = b - off
        buf[s:s + L] = pat
        count += 1
    return bytes(buf), count


# ------------------------------------------------------------------ C5 jobs
@dataclass
class Job:
    job_id: int
    data: bytes
    pairs: List[Pair]


def c5_job(job_id: int, min_size: int = 4096, max_size: int = 64 * MiB, seed: int = 5) -> Job:
    rng = np.random.default_rng([seed, job_id])
    size = int(np.exp(rng.uniform(np.log(min_size), np.log(max_size))))
    k = int(rng.integers(4, 65))
    alphabet = rng.choice(256, size=k, replace=False).astype(np.uint8)
    data = alphabet[rng.integers(0, k, size=size)].tobytes()
    pairs = []
    for _ in range(int(rng.integers(1, 17))):
        L = int(rng.integers(1, 33))
        if rng.random() < 0.6 and size > L:
            s = int(rng.integers(0, size - L))
            pat = data[s:s + L]
        else:
            pat = alphabet[rng.integers(0, k, size=L)].tobytes()
        R = int(rng.integers(0, 65))
        rep = rng.integers(0, 256, size=R, dtype=np.uint8).tobytes()
        pairs.append((pat, rep))
    return Job(job_id, data, pairs)
