"""The C-ABI library loads and exports every entry point declared in include/*.h.
CPU only: no call here touches a GPU."""
import ctypes
import re
import subprocess
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
REFERENCE_EXPORTS = {
    "cuda_replace_unified", "cuda_free_host", "cuda_replace_open", "cuda_replace_reset",
    "cuda_replace_build_index", "cuda_replace_apply", "cuda_replace_apply_seeded",
    "cuda_replace_query_prefix", "cuda_replace_apply_batch", "cuda_replace_result",
    "cuda_replace_close", "cuda_replace_version",
}


def declared_functions():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(cuda_\w+)\s*\(", text))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}


def test_header_declares_reference_abi():
    assert REFERENCE_EXPORTS <= declared_functions()


def test_library_exports_every_declared_symbol(cr_lib):
    exported = exported_symbols(cr_lib.path)
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    # nothing but the C ABI is visible
    assert {s for s in exported if not s.startswith("cuda_")} == set()


def test_library_loads_and_reports_version(cr_lib):
    v = cr_lib.version()
    assert "cuda_replace_b200" in v and "sm_100a" in v


def test_library_is_built_for_sm100a():
    from cuda_replace_b200 import build as B
    assert B.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]
    lib = ctypes.CDLL(str(B.LIB_PATH))
    assert lib.cuda_replace_open is not None


def test_host_copy_fills_new_bytes(cr_lib):
    """cuda_replace_host_copy is plain host memory work (no GPU): large results are copied
    into an uninitialised bytes object on several threads."""
    import random
    from cuda_replace_b200 import cuda_replace_wrapper as Wr
    n = (9 << 20) + 12345
    src = (ctypes.c_uint8 * n).from_buffer(bytearray(random.Random(1).randbytes(n)))
    out = Wr._bytes_at(ctypes.cast(src, Wr.c_uint8_p), n, cr_lib.lib)
    assert isinstance(out, bytes) and out == bytes(src)
    small = Wr._bytes_at(ctypes.cast(src, Wr.c_uint8_p), 1000, cr_lib.lib)
    assert small == bytes(src)[:1000]
