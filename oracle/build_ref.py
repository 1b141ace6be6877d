"""TEST INFRASTRUCTURE ONLY: build the reference library for sm_100a as a second checker.

Recipe: copy the reference source ``cuda_replace.cu`` (RAZZULLIX/cuda_replace) into
``oracle/_ref/`` (git-ignored, never committed), apply a purely mechanical patch, and
compile it with nvcc into ``oracle/_ref/libcuda_replace_ref.so``. The reference's ctypes
wrapper ``cuda_replace_wrapper.py`` is copied beside it unchanged, so the GPU parity tests
drive both libraries through the reference's own binding.

The reference checkout is read from ``--ref-dir DIR``, else from the environment variable
``CUDA_REPLACE_REF_DIR``, else from ``/root/reference`` (where this build machine mounts it).

Why a patch is needed: the reference's error macros jump with ``goto cuda_fail`` over
initialised local declarations (e.g. cuda_replace.cu:370-371, 1013, 1051), which MSVC
accepts and nvcc's front end rejects with "transfer of control bypasses initialization".
The patch only moves initialisers: ``T *a = x, *b = y;`` becomes ``T *a; T *b; a = x; b =
y;`` on the same line (``const`` dropped), and the two ``dim3`` locals of
query_kept_prefix (cuda_replace.cu:1850-1851) are declared at the top of that function.
The compiler itself names every declaration to patch, so no line list is hard-coded.
Nothing else in the reference changes; the library keeps all 12 exports.

The built library is a GPU library: it runs only where a GPU is present, and only on
inputs inside its envelope (n, kept and output below 2**31).
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_DIR = Path(os.environ.get("CUDA_REPLACE_REF_DIR", "/root/reference"))
REF_SRC = REF_DIR / "cuda_replace.cu"
OUT_DIR = HERE / "_ref"
PATCHED = OUT_DIR / "cuda_replace_ref.cu"
LIB = OUT_DIR / "libcuda_replace_ref.so"
WRAPPER = OUT_DIR / "cuda_replace_wrapper.py"
NVCC_FLAGS = ["-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
              "-gencode", "arch=compute_100a,code=sm_100a"]

_BYPASS = re.compile(r'variable "(\w+)" \(declared at line (\d+)\)')


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _compile(src: Path, out: Path) -> str:
    r = subprocess.run([_nvcc(), *NVCC_FLAGS, "-o", str(out), str(src)],
                       capture_output=True, text=True)
    return "" if r.returncode == 0 else (r.stdout + r.stderr)


def _split_top_level(s: str) -> list[str]:
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def _statement_span(lines: list[str], start: int) -> int:
    """Index of the line holding the ';' that ends the declaration starting at start."""
    depth = 0
    for i in range(start, len(lines)):
        code = lines[i].split("//", 1)[0]
        for ch in code:
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == ";" and depth == 0:
                return i
    raise ValueError(f"unterminated declaration at line {start + 1}")


def _patch_decl(lines: list[str], idx: int) -> None:
    end = _statement_span(lines, idx)
    text = " ".join(l.split("//", 1)[0].strip() for l in lines[idx:end + 1])
    indent = re.match(r"\s*", lines[idx]).group(0)
    m = re.match(r"(?:const\s+)?([A-Za-z_][\w:]*)\s+(.*);\s*$", text)
    if not m:
        raise ValueError(f"cannot parse declaration at line {idx + 1}: {text}")
    typ, rest = m.group(1), m.group(2)
    if typ == "dim3":
        # class type: declare at the top of the enclosing function, assign in place
        name, args = re.match(r"(\w+)\s*\((.*)\)\s*$", rest).groups()
        j = idx
        while not lines[j].startswith("{"):  # the function body opens at column 0
            j -= 1
        lines[j] = lines[j].rstrip() + f" dim3 {name};"
        lines[idx] = f"{indent}{name} = dim3({args});"
    else:
        decls, assigns = [], []
        for d in _split_top_level(rest):
            dm = re.match(r"\s*(\**)\s*(\w+)\s*=\s*(.*?)\s*$", d, re.S)
            if not dm:
                raise ValueError(f"cannot parse declarator '{d}' at line {idx + 1}")
            stars, name, init = dm.groups()
            decls.append(f"{typ} {stars}{name};")
            assigns.append(f"{name} = {init};")
        lines[idx] = indent + " ".join(decls + assigns)
    for k in range(idx + 1, end + 1):  # keep line numbers stable
        lines[k] = ""


def _copy_wrapper(ref_dir: Path) -> None:
    src = ref_dir / "cuda_replace_wrapper.py"
    if src.exists() and (not WRAPPER.exists() or WRAPPER.read_bytes() != src.read_bytes()):
        shutil.copyfile(src, WRAPPER)


def build_reference(force: bool = False, verbose: bool = True, ref_dir: Path | None = None) -> Path:
    ref_dir = Path(ref_dir) if ref_dir is not None else REF_DIR
    ref_src = ref_dir / "cuda_replace.cu"
    if LIB.exists() and not force:
        if ref_dir.exists():
            _copy_wrapper(ref_dir)
        return LIB
    if not ref_src.exists():
        raise FileNotFoundError(f"reference source not found: {ref_src}")
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    _copy_wrapper(ref_dir)
    lines = ref_src.read_text().split("\n")
    for _ in range(6):
        PATCHED.write_text("\n".join(lines))
        err = _compile(PATCHED, LIB)
        if not err:
            if verbose:
                print(f"built {LIB}")
            return LIB
        targets = sorted({int(l) for _, l in _BYPASS.findall(err)}, reverse=True)
        if not targets:
            raise RuntimeError("reference build failed for another reason:\n" + err[-4000:])
        done = set()
        for line_no in targets:
            if line_no in done:
                continue
            _patch_decl(lines, line_no - 1)
            done.add(line_no)
    raise RuntimeError("reference build did not converge")


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--ref-dir", default=None, help="reference checkout (holds cuda_replace.cu)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build_reference(force=a.force, ref_dir=Path(a.ref_dir) if a.ref_dir else None)
