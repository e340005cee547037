"""The plugin micro-kernels: drop-ins for the reference's native core.

Each function has the name, positional arguments, validation order, error
messages and output layout of its PyO3 counterpart in
native/core/src/lib.rs (the module that python/blackhole_sim/native_kernels.py
binds through ``importlib.import_module("blackhole_native")``):

* sequence / ndarray arguments return a flat Python ``list`` like the Rust
  ``Vec<f64>`` results;
* CUDA ``torch.Tensor`` arguments stay on the device and return a tensor
  (the zero-copy fast path).

The float64 results equal the reference's bit for bit.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _device as dev
from . import _lib

COEFFS_PER_CELL = 11
STOKES_COMPONENTS = 4


# ---------------------------------------------------------------- validation
def _ds(ds_cm) -> float:
    ds = float(ds_cm)
    if not math.isfinite(ds) or ds < 0.0:  # lib.rs:229-233, :318-322
        raise ValueError("ds_cm must be finite and non-negative")
    return ds


def _validate_grid(name: str, g: np.ndarray) -> None:  # lib.rs:112-129
    if g.size < 2:
        raise ValueError(f"{name} grid must contain at least 2 values")
    if not np.all(np.isfinite(g)):
        raise ValueError(f"{name} grid must contain only finite values")
    if np.any(g[1:] <= g[:-1]):
        raise ValueError(f"{name} grid must be strictly increasing")


def _validate_sampler_host(coeffs, rg, tg, pg, points) -> int:  # lib.rs:131-169
    _validate_grid("r", rg)
    _validate_grid("theta", tg)
    _validate_grid("phi", pg)
    if not np.all(np.isfinite(coeffs)):
        raise ValueError("coeffs must contain only finite values")
    expected = rg.size * tg.size * pg.size * COEFFS_PER_CELL
    if coeffs.size != expected:
        raise ValueError(f"coeffs must contain exactly r*theta*phi*11 values; expected {expected}, got {coeffs.size}")
    if points.size % 3 != 0:
        raise ValueError("points must contain flat r, theta, phi triples")
    if not np.all(np.isfinite(points)):
        raise ValueError("points must contain only finite values")
    return points.size // 3


def _validate_grid_device(name: str, g: torch.Tensor) -> None:
    if g.numel() < 2:
        raise ValueError(f"{name} grid must contain at least 2 values")
    bad, nonmono = dev.check_values_device(g, True)
    if bad:
        raise ValueError(f"{name} grid must contain only finite values")
    if nonmono:
        raise ValueError(f"{name} grid must be strictly increasing")


def _validate_sampler_device(coeffs, rg, tg, pg, points) -> int:
    _validate_grid_device("r", rg)
    _validate_grid_device("theta", tg)
    _validate_grid_device("phi", pg)
    if dev.check_values_device(coeffs, False)[0]:
        raise ValueError("coeffs must contain only finite values")
    expected = rg.numel() * tg.numel() * pg.numel() * COEFFS_PER_CELL
    if coeffs.numel() != expected:
        raise ValueError(
            f"coeffs must contain exactly r*theta*phi*11 values; expected {expected}, got {coeffs.numel()}")
    if points.numel() % 3 != 0:
        raise ValueError("points must contain flat r, theta, phi triples")
    if dev.check_values_device(points, False)[0]:
        raise ValueError("points must contain only finite values")
    return points.numel() // 3


def _dev_f64(x, device) -> torch.Tensor:
    return x.detach().to(device=device, dtype=torch.float64).contiguous().reshape(-1)


def _any_cuda(*xs) -> bool:
    return any(dev.is_cuda_tensor(x) for x in xs)


# ---------------------------------------------------------------- kernels
def stokes_rk2_brick(coeffs, ds_cm, initial):
    """One RK2 Stokes step per coefficient cell (native/core/src/lib.rs:227-279).

    coeffs: flat cells*11 values; initial: 4 (broadcast) or 4*cells values.
    Returns the flat cells*4 stepped Stokes values.
    """
    return _stokes_brick(coeffs, ds_cm, initial, "bhn_stokes_rk2_brick")


def stokes_exact_brick(coeffs, ds_cm, initial):
    """One exact constant-coefficient Stokes step per coefficient cell: the
    augmented matrix exponential of polarized_transfer.stokes_step_exact
    (python/blackhole_sim/polarized_transfer.py:51-70), batched over cells,
    with the inputs and validation of stokes_rk2_brick."""
    return _stokes_brick(coeffs, ds_cm, initial, "bhn_stokes_exact_brick")


def _stokes_brick(coeffs, ds_cm, initial, entry):
    ds = _ds(ds_cm)
    if _any_cuda(coeffs, initial):
        device = dev.require_cuda()
        c = _dev_f64(torch.as_tensor(coeffs), device)
        if c.numel() == 0 or c.numel() % COEFFS_PER_CELL:
            raise ValueError("coeffs must contain one or more flat 11-coefficient cells")
        if dev.check_values_device(c, False)[0]:
            raise ValueError("coeffs must contain only finite values")
        cells = c.numel() // COEFFS_PER_CELL
        ini = _dev_f64(torch.as_tensor(initial), device)
        if ini.numel() != STOKES_COMPONENTS and ini.numel() != cells * STOKES_COMPONENTS:
            raise ValueError("initial must contain either 4 values or 4 values per coefficient cell")
        if dev.check_values_device(ini, False)[0]:
            raise ValueError("initial must contain only finite values")
        out = torch.empty(cells * STOKES_COMPONENTS, dtype=torch.float64, device=device)
        _lib.check(getattr(_lib.lib(), entry)(dev.ptr(c), cells, ds, dev.ptr(ini), ini.numel(), dev.ptr(out),
                                              dev.stream_ptr()))
        return out
    c = dev.host_f64(coeffs)
    if c.size == 0 or c.size % COEFFS_PER_CELL:
        raise ValueError("coeffs must contain one or more flat 11-coefficient cells")
    if not np.all(np.isfinite(c)):
        raise ValueError("coeffs must contain only finite values")
    cells = c.size // COEFFS_PER_CELL
    ini = dev.host_f64(initial)
    if ini.size != STOKES_COMPONENTS and ini.size != cells * STOKES_COMPONENTS:
        raise ValueError("initial must contain either 4 values or 4 values per coefficient cell")
    if not np.all(np.isfinite(ini)):
        raise ValueError("initial must contain only finite values")
    device = dev.require_cuda()
    dc, di = dev.to_device_many((c, ini), device)
    out = torch.empty(cells * STOKES_COMPONENTS, dtype=torch.float64, device=device)
    _lib.check(getattr(_lib.lib(), entry)(dev.ptr(dc), cells, ds, dev.ptr(di), ini.size, dev.ptr(out),
                                          dev.stream_ptr()))
    return out.cpu().numpy().tolist()


def sample_brick_trilinear(coeffs, r_grid, theta_grid, phi_grid, points):
    """Trilinear coefficient samples (native/core/src/lib.rs:281-306).

    Returns flat n*11 values, NaN rows outside the nonperiodic r/theta domain.
    """
    if _any_cuda(coeffs, r_grid, theta_grid, phi_grid, points):
        device = dev.require_cuda()
        c, rg, tg, pg, pts = (_dev_f64(torch.as_tensor(x), device) for x in (coeffs, r_grid, theta_grid, phi_grid, points))
        n = _validate_sampler_device(c, rg, tg, pg, pts)
        out = torch.empty(n * COEFFS_PER_CELL, dtype=torch.float64, device=device)
        _launch_sample_trilinear(c, rg, tg, pg, pts, n, out)
        return out
    c, rg, tg, pg, pts = (dev.host_f64(x) for x in (coeffs, r_grid, theta_grid, phi_grid, points))
    n = _validate_sampler_host(c, rg, tg, pg, pts)
    device = dev.require_cuda()
    d = dev.to_device_many((c, rg, tg, pg, pts), device)
    out = torch.empty(n * COEFFS_PER_CELL, dtype=torch.float64, device=device)
    _launch_sample_trilinear(*d, n, out)
    return out.cpu().numpy().tolist()


def sample_and_step_stokes(coeffs, r_grid, theta_grid, phi_grid, points, ds_cm, initial, invalid_policy="nan"):
    """Sample then one RK2 Stokes step (native/core/src/lib.rs:308-366).

    The reference's native function takes no policy and returns NaN rows for
    out-of-domain samples (the default here); the optional ``invalid_policy``
    ('nan', 'initial', 'zero') applies native_kernels.py:342-350 on the device.
    Returns flat n*4 values.
    """
    ds = _ds(ds_cm)
    if invalid_policy not in _lib.POLICY_CODES:
        raise ValueError("invalid_policy must be 'nan', 'initial', or 'zero'")
    policy = _lib.POLICY_CODES[invalid_policy]
    if _any_cuda(coeffs, r_grid, theta_grid, phi_grid, points, initial):
        device = dev.require_cuda()
        c, rg, tg, pg, pts = (_dev_f64(torch.as_tensor(x), device) for x in (coeffs, r_grid, theta_grid, phi_grid, points))
        n = _validate_sampler_device(c, rg, tg, pg, pts)
        ini = _dev_f64(torch.as_tensor(initial), device)
        if ini.numel() != STOKES_COMPONENTS and ini.numel() != n * STOKES_COMPONENTS:
            raise ValueError("initial must contain either 4 values or 4 values per sample point")
        if dev.check_values_device(ini, False)[0]:
            raise ValueError("initial must contain only finite values")
        out = torch.empty(n * STOKES_COMPONENTS, dtype=torch.float64, device=device)
        _launch_sample_and_step(c, rg, tg, pg, pts, n, ds, ini, policy, out)
        return out
    c, rg, tg, pg, pts = (dev.host_f64(x) for x in (coeffs, r_grid, theta_grid, phi_grid, points))
    n = _validate_sampler_host(c, rg, tg, pg, pts)
    ini = dev.host_f64(initial)
    if ini.size != STOKES_COMPONENTS and ini.size != n * STOKES_COMPONENTS:
        raise ValueError("initial must contain either 4 values or 4 values per sample point")
    if not np.all(np.isfinite(ini)):
        raise ValueError("initial must contain only finite values")
    device = dev.require_cuda()
    d = dev.to_device_many((c, rg, tg, pg, pts, ini), device)
    out = torch.empty(n * STOKES_COMPONENTS, dtype=torch.float64, device=device)
    _launch_sample_and_step(*d[:5], n, ds, d[5], policy, out)
    return out.cpu().numpy().tolist()


SORT_MIN_POINTS = 1 << 18   # from this many points the sampler takes them in brick-cell order


def _launch_sample_and_step(c, rg, tg, pg, pts, n: int, ds: float, ini, policy: int, out) -> None:
    """bhn_sample_and_step_stokes, or for large point sets its cell-ordered form
    (bhn_sample_and_step_stokes_sorted: the same values, neighbouring points
    sharing cached corners); every argument already on the device."""
    L = _lib.lib()
    args = (dev.ptr(c), dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(), dev.ptr(pg), pg.numel(), dev.ptr(pts), n, ds,
            dev.ptr(ini), ini.numel(), policy, dev.ptr(out))
    nbytes = int(L.bhn_sample_sort_scratch_bytes(n, rg.numel() * tg.numel() * pg.numel())) if n >= SORT_MIN_POINTS \
        else -1
    if nbytes <= 0:
        _lib.check(L.bhn_sample_and_step_stokes(*args, dev.stream_ptr()))
        return
    scratch = torch.empty(nbytes + 256, dtype=torch.uint8, device=out.device)
    sp = (dev.ptr(scratch) + 255) & ~255
    _lib.check(L.bhn_sample_and_step_stokes_sorted(*args, sp, nbytes, dev.stream_ptr()))


def _launch_sample_trilinear(c, rg, tg, pg, pts, n: int, out) -> None:
    """bhn_sample_brick_trilinear, in cell order for large point sets (same values)."""
    L = _lib.lib()
    args = (dev.ptr(c), dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(), dev.ptr(pg), pg.numel(), dev.ptr(pts), n,
            dev.ptr(out))
    nbytes = int(L.bhn_sample_sort_scratch_bytes(n, rg.numel() * tg.numel() * pg.numel())) if n >= SORT_MIN_POINTS \
        else -1
    if nbytes <= 0:
        _lib.check(L.bhn_sample_brick_trilinear(*args, dev.stream_ptr()))
        return
    scratch = torch.empty(nbytes + 256, dtype=torch.uint8, device=out.device)
    sp = (dev.ptr(scratch) + 255) & ~255
    _lib.check(L.bhn_sample_brick_trilinear_sorted(*args, sp, nbytes, dev.stream_ptr()))


def sample_brick_valid_mask(r_grid, theta_grid, points):
    """True for points inside the inclusive nonperiodic r/theta domain, phi
    ignored (native_kernels.py:189-210).  Points may be flat triples or (n, 3)."""
    if _any_cuda(r_grid, theta_grid, points):
        device = dev.require_cuda()
        rg, tg, pts = (_dev_f64(torch.as_tensor(x), device) for x in (r_grid, theta_grid, points))
        _validate_grid_device("r", rg)
        _validate_grid_device("theta", tg)
        if pts.numel() % 3:
            raise ValueError("points must contain r/theta/phi triples")  # native_kernels.py:86-87
        if dev.check_values_device(pts, False)[0]:
            raise ValueError("points must contain only finite values")
        n = pts.numel() // 3
        mask = torch.empty(n, dtype=torch.uint8, device=device)
        _lib.check(_lib.lib().bhn_sample_brick_valid_mask(dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(),
                                                          dev.ptr(pts), n, dev.ptr(mask), dev.stream_ptr()))
        return mask.bool()
    rg, tg, pts = (dev.host_f64(x) for x in (r_grid, theta_grid, points))
    _validate_grid("r", rg)
    _validate_grid("theta", tg)
    if pts.size % 3:
        raise ValueError("points must contain r/theta/phi triples")  # native_kernels.py:86-87
    if not np.all(np.isfinite(pts)):
        raise ValueError("points must contain only finite values")
    n = pts.size // 3
    device = dev.require_cuda()
    d = dev.to_device_many((rg, tg, pts), device)
    mask = torch.empty(n, dtype=torch.uint8, device=device)
    _lib.check(_lib.lib().bhn_sample_brick_valid_mask(dev.ptr(d[0]), rg.size, dev.ptr(d[1]), tg.size, dev.ptr(d[2]),
                                                      n, dev.ptr(mask), dev.stream_ptr()))
    return [bool(v) for v in mask.cpu().numpy()]
