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


def to_device_many(arrays, device: torch.device) -> list[torch.Tensor]:
    """Several float64 host arrays -> device tensors.  Up to 8 MB together they
    go in one host-to-device copy, packed back to back (each start 32-byte
    aligned) and returned as views of one device buffer."""
    flats = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in arrays]
    if sum(f.nbytes for f in flats) > (8 << 20):  # large inputs: one copy each, no host repacking
        return [to_device(f, device) for f in flats]
    offs, total = [], 0
    for f in flats:
        offs.append(total)
        total += -(-f.size // 4) * 4
    host = np.empty(max(total, 1), dtype=np.float64)
    for f, o in zip(flats, offs):
        host[o:o + f.size] = f
    buf = to_device(host, device)
    return [buf[o:o + f.size] for f, o in zip(flats, offs)]


def check_values_device(t: torch.Tensor, increasing: bool) -> tuple[int, int]:
    """(non-finite count, non-increasing neighbour count) of a float64 device tensor."""
    counts = torch.zeros(2, dtype=torch.int32, device=t.device)
    _lib.check(_lib.lib().bhn_check_values(ptr(t), t.numel(), int(bool(increasing)), ptr(counts), stream_ptr()))
    c = counts.cpu().tolist()
    return int(c[0]), int(c[1])
