"""cuda_replace_stream_fd: chained replacement from one file descriptor to another, chunk-major
on the device, the input read and the output written piece by piece. The result must equal the
chained bytes.replace for any chunk size, matches planted across every chunk boundary included
(the reference's pair-major helper drops those, cuda_replace_wrapper.py:356)."""
import os
import tempfile
import threading

import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu

MiB = 1 << 20


def chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


@pytest.mark.parametrize("chunk", [4096, 1 * MiB, 3 * MiB + 17])
def test_file_to_file(cr_lib, chunk):
    buf, pairs, planted = WL.c4_input(24 * MiB + 321, chunk=chunk if chunk > 4096 else MiB, seed=4)
    data = bytes(buf)
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in"), os.path.join(d, "out")
        with open(src, "wb") as f:
            f.write(data)
        with open(src, "rb") as fi, open(dst, "wb") as fo:
            nin, nout = Wr.stream_file(cr_lib, fi.fileno(), fo.fileno(), pairs, chunk)
        with open(dst, "rb") as f:
            got = f.read()
    want = chain(data, pairs)
    assert nin == len(data) and nout == len(want) and got == want


def test_pipe_in_and_empty_input(cr_lib):
    """The input's end is found by reading ahead, so a pipe works; an empty input writes nothing."""
    data = WL.text_corpus(5 * MiB + 3, seed=4)
    pairs = WL.c4_pairs(4)
    r, w = os.pipe()

    def feed():
        with os.fdopen(w, "wb") as f:
            for i in range(0, len(data), 65536):
                f.write(data[i:i + 65536])

    t = threading.Thread(target=feed)
    t.start()
    with tempfile.TemporaryFile() as fo:
        nin, nout = Wr.stream_file(cr_lib, r, fo.fileno(), pairs, MiB)
        t.join()
        os.close(r)
        fo.seek(0)
        got = fo.read()
    assert nin == len(data) and got == chain(data, pairs) and nout == len(got)
    with tempfile.TemporaryFile() as fi, tempfile.TemporaryFile() as fo:
        assert Wr.stream_file(cr_lib, fi.fileno(), fo.fileno(), pairs, MiB) == (0, 0)
