"""The presence index (cuda_replace_build_index): the next apply skips the candidate search in
16 KiB sub-tiles whose chunk lacks the pattern's first byte. Results must not change, and any
change of the buffer must retire the index. The reference builds such an index and never reads
it (cuda_replace.cu:398-442, 2320-2354)."""
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


@pytest.mark.parametrize("chunk", [None, 16384, 50000, 1 << 20, 4 << 20])
def test_index_keeps_results(cr_lib, chunk):
    """Sparse needles in Zipf text (their first byte occurs in few chunks), at chunk sizes from
    the 16 KiB minimum up; apply, apply_seeded and apply_batch after build_index."""
    rng = random.Random(chunk or 1)
    txt = bytearray(WL.text_corpus(24 * MiB + 777, seed=3))
    for _ in range(40):
        pos = rng.randrange(len(txt) - 16)
        txt[pos:pos + 6] = b"NEEDLE"
    for pos in (16384 - 3, 65536 - 1, (1 << 20) - 2, (4 << 20) - 5, len(txt) - 6):  # across boundaries
        txt[pos:pos + 6] = b"NEEDLE"
    src = bytes(txt)
    for pairs in ([(b"NEEDLE", b"FOUND")], [(b"NEEDLE", b"")], [(b"NEEDLE", b"X" * 20)],
                  [(b"NEEDLE", b"Q"), (b"QQ", b"w"), (b"the ", b"THE ")]):
        with Wr.Session(cr_lib, src) as s:
            s.build_index(chunk)
            if len(pairs) == 1:
                s.apply(*pairs[0])
            else:
                s.apply_batch(pairs)
            assert s.result() == chain(src, pairs)
    with Wr.Session(cr_lib, src) as s:
        s.build_index(chunk)
        n, last = s.apply_seeded(b"NEEDLE", b"F", 3)  # candidates before 3 + 6 are not taken
        got = s.result()
        assert n == len(got) and got == src[:9] + src[9:].replace(b"NEEDLE", b"F")


def test_index_retired_when_the_buffer_changes(cr_lib):
    """An index of the buffer before an apply must not be used after it: the first apply here
    creates the only occurrences of the second pattern's first byte."""
    src = b"xy" * (3 * MiB) + b"ab" + b"xy" * 1000
    with Wr.Session(cr_lib, src) as s:
        s.build_index()
        s.apply(b"ab", b"Nx")
        s.apply(b"Nx", b"Q")
        assert s.result() == src.replace(b"ab", b"Nx").replace(b"Nx", b"Q")
        s.build_index(16384)
        s.reset(src)
        s.apply(b"ab", b"Z")
        assert s.result() == src.replace(b"ab", b"Z")
