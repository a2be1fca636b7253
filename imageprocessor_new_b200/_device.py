"""Device buffers and streams for the C ABI: torch tensors used as plain CUDA allocations."""

from __future__ import annotations

import contextlib
import os

import numpy as np
import torch

from . import _lib


def device(index: int = 0) -> torch.device:
    return torch.device("cuda", int(index))


@contextlib.contextmanager
def on_device(index: int = 0):
    """Makes CUDA device ``index`` current (subpx/backends.py:55-59 gpu_device)."""
    _lib.lib()
    with torch.cuda.device(int(index)):
        yield


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


_UPLOAD_POOL = None
_UPLOAD_CHUNK = 8 << 20  # bytes per host copy / device copy pair of a large upload


def _upload_pool():
    global _UPLOAD_POOL
    if _UPLOAD_POOL is None:
        from concurrent.futures import ThreadPoolExecutor

        _UPLOAD_POOL = ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)),
                                          thread_name_prefix="spx-upload")
    return _UPLOAD_POOL


def upload(a: np.ndarray) -> torch.Tensor:
    """Host array -> contiguous device tensor (same dtype), queued on the current stream.

    The data goes through pinned memory: a copy from pageable memory would first synchronise the
    stream (draining the GPU at every small upload); from pinned memory it is asynchronous, and
    torch's host allocator keeps the pinned block until the copy has run. A large array is copied
    into the pinned block in 8 MB chunks by a few host threads, and each chunk's device copy is
    queued as soon as its host copy is done, so the two overlap."""
    a = np.ascontiguousarray(a)
    dtype = TORCH_ALL.get(a.dtype) or torch.from_numpy(np.empty(0, a.dtype)).dtype
    pinned = torch.empty(a.shape, dtype=dtype, pin_memory=True)
    if a.nbytes < 4 * _UPLOAD_CHUNK:
        pinned.numpy()[...] = a
        return pinned.to("cuda", non_blocking=True)
    out = torch.empty(a.shape, dtype=dtype, device="cuda")
    n = a.nbytes
    src = a.reshape(-1).view(np.uint8)
    host = pinned.numpy().reshape(-1).view(np.uint8)
    host_t = pinned.view(-1).view(torch.uint8)
    dev_t = out.view(-1).view(torch.uint8)
    bounds = [(lo, min(lo + _UPLOAD_CHUNK, n)) for lo in range(0, n, _UPLOAD_CHUNK)]

    def copy(lo, hi):
        host[lo:hi] = src[lo:hi]  # NumPy releases the GIL for the copy

    pool = _upload_pool()
    futures = [pool.submit(copy, lo, hi) for lo, hi in bounds]
    for (lo, hi), f in zip(bounds, futures):
        f.result()
        dev_t[lo:hi].copy_(host_t[lo:hi], non_blocking=True)
    return out


def start_download(t: torch.Tensor) -> np.ndarray:
    """Queues a copy of a device tensor into pinned host memory on the current stream and returns
    the host array; its contents are valid once the stream has been synchronised."""
    host = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    host.copy_(t, non_blocking=True)
    return host.numpy()


def empty(shape, dtype) -> torch.Tensor:
    return torch.empty(shape, dtype=dtype, device="cuda")


def workspace(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def read_int(t: torch.Tensor) -> int:
    """Value of a one-element device int tensor (synchronises the stream)."""
    return int(t.item())


TORCH_DTYPES = {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
                np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}
# Every dtype the package uploads (image dtypes plus indices, flags and parameters).
TORCH_ALL = {**TORCH_DTYPES, np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16,
             np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64, np.dtype(np.bool_): torch.bool,
             np.dtype(np.uint32): torch.uint32, np.dtype(np.uint64): torch.uint64}


def dtype_code(t: torch.Tensor) -> int:
    for np_dtype, torch_dtype in TORCH_DTYPES.items():
        if t.dtype == torch_dtype:
            return _lib.DTYPES[np_dtype]
    raise ValueError(f"unsupported image dtype {t.dtype}")
