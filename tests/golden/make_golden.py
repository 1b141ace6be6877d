"""Generate tests/golden/vectors.json: known-answer vectors for the replace path.

Expected values come from CPython ``bytes.replace`` (chained per pair), the ground truth
the reference checks itself against (test/test.py:150-161). Inputs are stored as recipes
(concatenated repeated units) or generator parameters, outputs as length + SHA-256 (plus
the full bytes when short). Sources of the cases:

* the reference's own benchmark cases (test/test.py:44-99) and wrapper self-test
  (cuda_replace_wrapper.py:379-392), and the README usage example (README.md:40-42);
* minimal vectors for the reference defects found in the survey of cuda_replace.cu
  (tile-carry composition cu:737-884, zero-filled halo cu:766, streaming truncation
  py:356, empty pattern cu:2104), whose expected value is bytes.replace;
* seeded cases (apply_seeded carry-in) and query_prefix answers, from the oracle
  restatement cross-checked here against a pure-Python greedy;
* scaled-down digests of the five benchmark configurations.

Run: ``python tests/golden/make_golden.py`` (writes vectors.json next to this file).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from cuda_replace_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

MiB = 1 << 20


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def recipe_bytes(recipe) -> bytes:
    return b"".join(bytes.fromhex(u) * c for u, c in recipe)


def case(name, recipe, pairs, source, keep_output=None):
    src = recipe_bytes(recipe)
    out = O.chain(src, pairs)
    d = {
        "name": name, "source": source, "recipe": recipe,
        "pairs": [[p.hex(), r.hex()] for p, r in pairs],
        "in_len": len(src), "out_len": len(out), "out_sha256": sha(out),
    }
    if keep_output or (keep_output is None and len(out) <= 256):
        d["out_hex"] = out.hex()
    return d


def h(b: bytes) -> str:
    return b.hex()


def known_answer():
    cases = [
        case("readme hello->goodbye", [[h(b"hello world hello universe"), 1]],
             [(b"hello", b"goodbye")], "README.md:40-42"),
        case("wrapper self-test aaa->X", [[h(b"aaabaaabaaa"), 1]], [(b"aaa", b"X")],
             "cuda_replace_wrapper.py:379-392"),
        case("test.py dense 1MB hello->hi", [[h(b"hello "), 1024 * 1024 // 6]], [(b"hello", b"hi")],
             "test/test.py:49-54"),
        case("test.py sparse 10MB NEEDLE", [[h(b"x"), 5 * MiB], [h(b"NEEDLE"), 1], [h(b"x"), 5 * MiB]],
             [(b"NEEDLE", b"FOUND")], "test/test.py:57-64"),
        case("test.py expansion 5MB abc->ABCDEF", [[h(b"abc"), 5 * MiB // 3]], [(b"abc", b"ABCDEF")],
             "test/test.py:67-72"),
        case("test.py medium 20MB REPLACE->DONE",
             [[h(b"normal text " * 100 + b"REPLACE "), 20 * 1024 // 12]], [(b"REPLACE", b"DONE")],
             "test/test.py:75-80"),
        case("test.py large 50MB aaa->X", [[h(b"aaabaaabaaab"), 50 * MiB // 12]], [(b"aaa", b"X")],
             "test/test.py:83-88"),
        case("test.py huge 100MB xx->y", [[h(b"x"), 100 * MiB]], [(b"xx", b"y")], "test/test.py:91-96"),
    ]
    return cases


def defect_vectors():
    return [
        case("D1 tile carry: 20000 x a, aaa->X", [[h(b"a"), 20000]], [(b"aaa", b"X")],
             "cuda_replace.cu:737-884 (tile-carry composition)", keep_output=False),
        case("D1 tile carry: 40001 x a, aaaaa->QR", [[h(b"a"), 40001]], [(b"aaaaa", b"QR")],
             "cuda_replace.cu:737-884", keep_output=False),
        case("D2 zero halo: xyza, a\\0->Q", [[h(b"xyza"), 1]], [(b"a\x00", b"Q")],
             "cuda_replace.cu:766, 839 (halo filled with zeros)"),
        case("D2 zero halo tail: ab\\0\\0 at end", [[h(b"zzab"), 1]], [(b"ab\x00\x00", b"")],
             "cuda_replace.cu:766"),
        case("D3 straddle: xxxaayyy aa->X", [[h(b"xxxaayyy"), 1]], [(b"aa", b"X")],
             "cuda_replace_wrapper.py:356 (chunk truncation)"),
        case("D5 empty pattern: abc, ''->-", [[h(b"abc"), 1]], [(b"", b"-")], "cuda_replace.cu:2104-2109"),
        case("D5 empty pattern on empty input", [], [(b"", b"xy")], "cuda_replace.cu:2104-2109"),
        case("empty input", [], [(b"a", b"b")], "edge"),
        case("pattern longer than input", [[h(b"ab"), 1]], [(b"abc", b"X")], "edge"),
        case("embedded NULs deletion", [[h(b"\x00\x00\x01\x00\x00\x00\x01\x01"), 3]],
             [(b"\x00\x00\x01", b"")], "single-pair workload shape: random 00 00 01 deleted"),
    ]


def seeded_vectors():
    """apply_seeded: (input, pat, rep, prev_last_rel) -> output, last kept, query answers."""
    rows = []
    cases = [
        (b"aaaaaaaaaa", b"aa", b"X", -1), (b"aaaaaaaaaa", b"aa", b"X", -2),
        (b"aaaaaaaaaa", b"aaa", b"Y", -1), (b"aaaaaaaaaa", b"aaa", b"Y", -2),
        (b"abababab", b"abab", b"Z", -3), (b"xxxaayyy", b"aa", b"", -1),
        (b"aaaa", b"aa", b"bcd", 0), (b"aaaaaaaa", b"aa", b"Q", 3),
        (b"hello world", b"lo", b"LO", -(1 << 29)),
    ]
    for src, pat, rep, seed in cases:
        bb = O.block_before_from_seed(seed, len(pat))
        out, kept, last = O.replace(src, pat, rep, bb)
        assert out == O.py_replace(src, pat, rep, bb)
        queries = []
        for lim in range(0, len(src) + 2):
            queries.append([lim, *O.query_prefix(src, pat, lim, bb)])
        rows.append({"src_hex": src.hex(), "pat_hex": pat.hex(), "rep_hex": rep.hex(), "prev_last_rel": seed,
                     "out_hex": out.hex(), "kept": kept, "last": last, "queries": queries})
    return rows


def config_inputs(row):
    """Regenerate the input and pairs of a config digest row (used by the tests too)."""
    g = row["generator"]
    if g["fn"] == "c1_acgt":
        d, p, r = W.c1_acgt(g["n"], seed=g["seed"])
        return d, [(p, r)]
    if g["fn"] == "c2_cases":
        name, gen, p, r = W.c2_cases(n_run=g["n_run"], n_rand=g["n_rand"], seed=g["seed"])[g["index"]]
        return gen(), [(p, r)]
    if g["fn"] == "text_corpus":
        return W.text_corpus(g["n"], seed=g["seed"]), W.c3_pairs(seed=g["seed"])
    raise ValueError(g["fn"])


def config_digests():
    gens = [{"fn": "c1_acgt", "n": 1 * MiB, "seed": 1, "name": "C1 scaled 1 MiB ACGT->N"}]
    for i, nm in enumerate(["aa->X", "a->bcd", "random 00 00 01->''"]):
        gens.append({"fn": "c2_cases", "index": i, "n_run": 3 * MiB + 5, "n_rand": 2 * MiB, "seed": 2,
                     "name": f"C2 scaled {nm}"})
    gens.append({"fn": "text_corpus", "n": 2 * MiB, "seed": 3, "name": "C3 scaled 2 MiB text x 128 pairs"})
    rows = []
    for g in gens:
        row = {"name": g.pop("name"), "source": "stated workload configurations (scaled)", "generator": g}
        src, pairs = config_inputs(row)
        out = O.chain(src, pairs)
        row.update({"in_len": len(src), "in_sha256": sha(src), "npairs": len(pairs),
                    "out_len": len(out), "out_sha256": sha(out)})
        rows.append(row)
    return rows


def main():
    O.build_oracle()
    doc = {
        "generated_by": "tests/golden/make_golden.py",
        "truth": "CPython bytes.replace, chained per pair",
        "known_answer": known_answer(),
        "defects": defect_vectors(),
        "seeded": seeded_vectors(),
        "configs": config_digests(),
    }
    (HERE / "vectors.json").write_text(json.dumps(doc, indent=1))
    print(f"wrote {HERE / 'vectors.json'}")


if __name__ == "__main__":
    main()
