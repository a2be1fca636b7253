"""Device buffers and streams for the C ABI: torch tensors used as plain CUDA allocations."""

from __future__ import annotations

import contextlib

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


def upload(a: np.ndarray) -> torch.Tensor:
    """Host array -> contiguous device tensor (same dtype)."""
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a).to("cuda", non_blocking=False)


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


def dtype_code(t: torch.Tensor) -> int:
    for np_dtype, torch_dtype in TORCH_DTYPES.items():
        if t.dtype == torch_dtype:
            return _lib.DTYPES[np_dtype]
    raise ValueError(f"unsupported image dtype {t.dtype}")
