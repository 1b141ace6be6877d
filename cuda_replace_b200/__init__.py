"""cuda_replace_b200: leftmost, non-overlapping byte-pattern replacement (bytes.replace
semantics) on NVIDIA B200, behind the C ABI of RAZZULLIX/cuda_replace.

The product is ``libcuda_replace.so`` (C ABI, include/cuda_replace.h); this package holds its
CUDA sources (csrc/), the in-tree build, and a ctypes binding with the reference wrapper's
interface (CudaReplaceLib, Session, replace_unified, gpu_replace_streaming), plus the batched
and served jobs (Server, replace_jobs).
"""
from .cuda_replace_wrapper import (  # noqa: F401
    DEFAULT_LIB,
    CudaReplaceLib,
    Server,
    Session,
    gpu_replace_streaming,
    replace_jobs,
    replace_unified,
)

__all__ = ["CudaReplaceLib", "Session", "replace_unified", "gpu_replace_streaming", "Server", "replace_jobs",
           "DEFAULT_LIB"]
