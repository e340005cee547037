"""Device plumbing: torch provides device memory and the current stream."""

from __future__ import annotations

import numpy as np
import torch

from . import _lib


def require_cuda() -> torch.device:
    """The current CUDA device; a RuntimeError when there is none (no CPU path exists)."""
    if not torch.cuda.is_available():
        raise RuntimeError("blackhole_native needs a CUDA GPU (sm_100a build); there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else int(t.data_ptr())


def is_cuda_tensor(x) -> bool:
    return isinstance(x, torch.Tensor) and x.is_cuda


def host_f64(x) -> np.ndarray:
    """Flat contiguous float64 host copy of a list / array / CPU tensor."""
    if isinstance(x, torch.Tensor):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))


def to_device(a: np.ndarray, device: torch.device) -> torch.Tensor:
    """Host array -> device tensor through pinned memory."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if t.numel() * t.element_size() >= (1 << 20):
        t = t.pin_memory()
    return t.to(device, non_blocking=True)


def check_values_device(t: torch.Tensor, increasing: bool) -> tuple[int, int]:
    """(non-finite count, non-increasing neighbour count) of a float64 device tensor."""
    counts = torch.zeros(2, dtype=torch.int32, device=t.device)
    _lib.check(_lib.lib().bhn_check_values(ptr(t), t.numel(), int(bool(increasing)), ptr(counts), stream_ptr()))
    c = counts.cpu().tolist()
    return int(c[0]), int(c[1])
