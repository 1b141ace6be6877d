"""Generate tests/golden/fullsize.json: digests of the chained bytes.replace output of three
workloads at their full stated sizes, for the GPU tests to compare against.

* the 128-pair chain: 4 GiB of tiled Zipf text (``workloads.c3_input``), 128 entity pairs;
* streaming: 16 GiB of tiled Zipf text with a pattern planted across every 256 MiB chunk
  boundary (``workloads.c4_input``), 8 mixed shrink/expand pairs;
* batched jobs: the first 1000 jobs of the 10,000-job generator (``workloads.c5_job``) at their
  full sizes (log-uniform 4 KiB-64 MiB), one (length, SHA-256) per job.

Ground truth is CPython ``bytes.replace``, chained per pair, as the reference checks itself
(test/test.py:150-161). Gigabytes of chained bytes.replace take minutes per core, so the
chains are computed piecewise on several processes: the input is cut right after occurrences
of a byte that no pattern and no replacement contains (a space for the entity pairs, a newline
for the streaming pairs, whose patterns end in a space). Such a byte is never removed (it
would have to lie inside a matched occurrence) and never created (no replacement holds it), so
no occurrence in any intermediate text spans a cut, the leftmost greedy carries no state
across one, and the chain of the whole input is the concatenation of the chains of the pieces.
The script checks the separator condition before it relies on it.

Run: ``python tests/golden/make_fullsize.py [c3] [c4] [c5]`` (all three by default); writes
fullsize.json next to this file. Takes several minutes and up to ~40 GB of host memory (c4).
"""
from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from cuda_replace_b200 import workloads as W  # noqa: E402

MiB = 1 << 20
GiB = 1 << 30
OUT = HERE / "fullsize.json"


def _chain(piece: bytes, pairs) -> bytes:
    for p, r in pairs:
        piece = piece.replace(p, r)
    return piece


def _piece_worker(args):
    piece, pairs = args
    return _chain(piece, pairs)


def cut_points(data, sep: int, piece: int):
    """Offsets just after an occurrence of byte `sep` near every multiple of `piece`."""
    cuts = [0]
    target = piece
    mv = memoryview(data)
    while target < len(data):
        j = bytes(mv[target:target + (1 << 20)]).find(bytes([sep]))
        if j < 0:
            j = data.find(bytes([sep]), target)
            if j < 0:
                break
        else:
            j += target
        cuts.append(j + 1)
        target = j + 1 + piece
    cuts.append(len(data))
    return sorted(set(cuts))


def chain_digest(data, pairs, sep: int, workers: int, piece: int = 256 * MiB):
    """(output length, SHA-256) of the chained bytes.replace of data, piecewise."""
    for p, r in pairs:
        assert sep not in p and sep not in r, "separator byte occurs in a pair"
    cuts = cut_points(data, sep, piece)
    mv = memoryview(data)
    spans = list(zip(cuts[:-1], cuts[1:]))
    h = hashlib.sha256()
    total = 0
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        pending = []  # at most 2 x workers pieces in flight (bounded host memory)
        nxt = 0
        for i in range(len(spans)):
            while nxt < len(spans) and len(pending) < 2 * workers:
                a, b = spans[nxt]
                pending.append(pool.apply_async(_piece_worker, ((bytes(mv[a:b]), pairs),)))
                nxt += 1
            out = pending.pop(0).get()
            h.update(out)
            total += len(out)
            del out
    return total, h.hexdigest(), len(spans)


def _job_worker(job_id: int):
    job = W.c5_job(job_id)
    out = _chain(job.data, job.pairs)
    return {"job_id": job_id, "in_len": len(job.data), "npairs": len(job.pairs),
            "out_len": len(out), "out_sha256": hashlib.sha256(out).hexdigest()}


def c3_row(workers):
    data, pairs = W.c3_input(4 * GiB, seed=3)
    n, d, pieces = chain_digest(data, pairs, ord(" "), workers)
    return {"name": "C3 4 GiB tiled text x 128 entity pairs", "generator": {"fn": "c3_input", "total": 4 * GiB, "seed": 3},
            "in_len": len(data), "in_sha256": hashlib.sha256(data).hexdigest(), "npairs": len(pairs),
            "out_len": n, "out_sha256": d, "pieces": pieces}


def c4_row(workers):
    data, pairs, planted = W.c4_input(16 * GiB, chunk=256 * MiB, seed=4)
    in_sha = hashlib.sha256(data).hexdigest()
    n, d, pieces = chain_digest(data, pairs, ord("\n"), workers)
    return {"name": "C4 16 GiB tiled text x 8 pairs, patterns planted across every 256 MiB boundary",
            "generator": {"fn": "c4_input", "total": 16 * GiB, "chunk": 256 * MiB, "seed": 4},
            "planted": planted, "in_len": len(data), "in_sha256": in_sha, "npairs": len(pairs),
            "out_len": n, "out_sha256": d, "pieces": pieces}


def c5_rows(workers, count=1000):
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        rows = list(pool.imap(_job_worker, range(count), chunksize=4))
    return rows


def main(argv):
    which = [a for a in argv if a in ("c3", "c4", "c5")] or ["c3", "c4", "c5"]
    workers = int(os.environ.get("GOLDEN_WORKERS", os.cpu_count() or 4))
    doc = json.loads(OUT.read_text()) if OUT.exists() else {}
    doc["generated_by"] = "tests/golden/make_fullsize.py"
    doc["truth"] = "CPython bytes.replace, chained per pair (computed piecewise at separator bytes)"
    for w in which:
        t0 = time.time()
        if w == "c3":
            doc["c3"] = c3_row(workers)
        elif w == "c4":
            doc["c4"] = c4_row(workers)
        else:
            doc["c5"] = {"name": "C5 first 1000 jobs at full size", "generator": {"fn": "c5_job", "seed": 5},
                         "jobs": c5_rows(workers)}
        print(f"{w}: {time.time() - t0:.1f} s", flush=True)
        OUT.write_text(json.dumps(doc, indent=1))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main(sys.argv[1:])
