"""CUDA stream plumbing: the C ABI takes a cudaStream_t as void*; by default
the library runs on torch's current stream so that it is ordered with torch
allocations and copies."""
from __future__ import annotations

import ctypes as C


def stream_handle(stream=None) -> C.c_void_p:
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)
