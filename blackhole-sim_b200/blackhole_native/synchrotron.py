"""Coefficient-brick precompute on the GPU.

Drop-in for ``precompute_coefficient_bricks`` (python/blackhole_sim/
coefficient_bricks.py:119-152) with the reference's synchrotron coefficient
models (python/blackhole_sim/synchrotron.py:240-325): the same arguments, the
same model parameters, the same ``[nr][ntheta][nphi][11]`` result in
``COEFF_NAMES`` order.  Every cell is computed by ``bhn_brick_precompute`` in
FP64 on the device; ``precompute_device_brick`` hands the result straight to
the renderer without a host round trip.

The snapshot and scaling arguments are duck-typed: any object with the
``GRMHDSnapshot`` fields (r, theta, phi, rho, theta_e, b_con, spin_a) and the
``PhysicalScaling`` fields (rho_cgs_per_code, b_gauss_per_code,
mean_molecular_weight_per_electron) works, the reference's own classes
included.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Literal

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .bricks import BrickGrid
from .render import DeviceBrick


@dataclass(frozen=True)
class ThermalSynchrotronCoefficients:
    """synchrotron.py:240-275 (Maxwell-Juettner electrons)."""

    gamma_grid_size: int = 192
    pitch_nodes: int = 16
    faraday_rotation_scale: float = 1.0
    faraday_conversion_scale: float = 1.0


@dataclass(frozen=True)
class NonthermalPowerLawSynchrotronCoefficients:
    """synchrotron.py:278-311 (power-law electrons)."""

    p: float = 3.5
    gamma_min: float = 10.0
    gamma_max: float = 1.0e5
    nonthermal_fraction: float = 0.02
    gamma_grid_size: int = 224
    pitch_nodes: int = 16
    absorption_scale: float = 1.0
    faraday_scale: float = 0.15


@dataclass(frozen=True)
class HybridSynchrotronCoefficients:
    """synchrotron.py:314-325: the sum of a thermal and a power-law component."""

    thermal: ThermalSynchrotronCoefficients = field(default_factory=ThermalSynchrotronCoefficients)
    nonthermal: NonthermalPowerLawSynchrotronCoefficients = field(
        default_factory=NonthermalPowerLawSynchrotronCoefficients)


class ModelStruct(ctypes.Structure):
    """``bhn_synchrotron_model``."""

    _fields_ = [
        ("nu_hz", ctypes.c_double),
        ("rho_cgs_per_code", ctypes.c_double),
        ("b_gauss_per_code", ctypes.c_double),
        ("mean_molecular_weight_per_electron", ctypes.c_double),
        ("thermal", ctypes.c_int32),
        ("nonthermal", ctypes.c_int32),
        ("thermal_gamma_n", ctypes.c_int32),
        ("thermal_pitch_n", ctypes.c_int32),
        ("thermal_rotation_scale", ctypes.c_double),
        ("thermal_conversion_scale", ctypes.c_double),
        ("nonthermal_gamma_n", ctypes.c_int32),
        ("nonthermal_pitch_n", ctypes.c_int32),
        ("nonthermal_p", ctypes.c_double),
        ("nonthermal_gamma_min", ctypes.c_double),
        ("nonthermal_gamma_max", ctypes.c_double),
        ("nonthermal_fraction", ctypes.c_double),
        ("nonthermal_absorption_scale", ctypes.c_double),
        ("nonthermal_faraday_scale", ctypes.c_double),
    ]


def _declare() -> ctypes.CDLL:
    L = _lib.lib()
    fn = L.bhn_brick_precompute
    vp = ctypes.c_void_p
    fn.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.POINTER(ModelStruct), vp, ctypes.c_int32, vp]
    fn.restype = ctypes.c_int
    return L


def model_struct(model, nu_hz: float, scaling) -> ModelStruct:
    """The C model for a Hybrid, Thermal or power-law model object (the
    reference's classes or this module's)."""
    m = ModelStruct()
    m.nu_hz = float(nu_hz)
    m.rho_cgs_per_code = float(scaling.rho_cgs_per_code)
    m.b_gauss_per_code = float(scaling.b_gauss_per_code)
    m.mean_molecular_weight_per_electron = float(getattr(scaling, "mean_molecular_weight_per_electron", 1.0))
    th = getattr(model, "thermal", None)
    nt = getattr(model, "nonthermal", None)
    if th is None and nt is None:  # a single component
        if hasattr(model, "faraday_rotation_scale"):
            th = model
        elif hasattr(model, "nonthermal_fraction"):
            nt = model
        else:
            raise TypeError("coeff_model must be a Hybrid, Thermal or NonthermalPowerLaw synchrotron model")
    if th is not None:
        m.thermal = 1
        m.thermal_gamma_n, m.thermal_pitch_n = int(th.gamma_grid_size), int(th.pitch_nodes)
        m.thermal_rotation_scale = float(th.faraday_rotation_scale)
        m.thermal_conversion_scale = float(th.faraday_conversion_scale)
    if nt is not None:
        m.nonthermal = 1
        m.nonthermal_gamma_n, m.nonthermal_pitch_n = int(nt.gamma_grid_size), int(nt.pitch_nodes)
        m.nonthermal_p, m.nonthermal_gamma_min, m.nonthermal_gamma_max = (float(nt.p), float(nt.gamma_min),
                                                                          float(nt.gamma_max))
        m.nonthermal_fraction = float(nt.nonthermal_fraction)
        m.nonthermal_absorption_scale = float(nt.absorption_scale)
        m.nonthermal_faraday_scale = float(nt.faraday_scale)
    return m


def _fields(snapshot, stride: int):
    if stride < 1:
        raise ValueError("stride must be >= 1")  # coefficient_bricks.py:133-134
    sl = (slice(None, None, stride),) * 3
    r = np.asarray(snapshot.r, dtype=np.float64)[::stride]
    theta = np.asarray(snapshot.theta, dtype=np.float64)[::stride]
    phi = np.asarray(snapshot.phi, dtype=np.float64)[::stride]
    rho = np.ascontiguousarray(np.asarray(snapshot.rho, dtype=np.float64)[sl])
    theta_e = np.ascontiguousarray(np.asarray(snapshot.theta_e, dtype=np.float64)[sl])
    b_con = np.ascontiguousarray(np.asarray(snapshot.b_con, dtype=np.float64)[sl])
    shape = (r.size, theta.size, phi.size)
    if rho.shape != shape or theta_e.shape != shape or b_con.shape != shape + (4,):
        raise ValueError(f"snapshot fields must have shape {shape} (b_con {shape + (4,)})")
    return r, theta, phi, rho, theta_e, b_con


def precompute_device_coefficients(snapshot, scaling, nu_hz: float = 230e9,
                                   dtype: Literal["float32", "float64"] = "float32", coeff_model=None,
                                   stride: int = 1, device: torch.device | None = None):
    """(r, theta, phi, coeffs) with coeffs a device tensor [nr][nt][np][11]."""
    if dtype not in ("float32", "float64"):
        raise ValueError("dtype must be 'float32' or 'float64'")
    L = _declare()
    device = device or dev.require_cuda()
    r, theta, phi, rho, theta_e, b_con = _fields(snapshot, stride)
    shape = (r.size, theta.size, phi.size)
    cells = int(np.prod(shape))
    d_rho = torch.from_numpy(rho).to(device)
    d_te = torch.from_numpy(theta_e).to(device)
    d_b = torch.from_numpy(b_con).to(device)
    tdt = torch.float32 if dtype == "float32" else torch.float64
    out = torch.empty(shape + (11,), dtype=tdt, device=device)
    m = model_struct(coeff_model or HybridSynchrotronCoefficients(), nu_hz, scaling)
    _lib.check(L.bhn_brick_precompute(dev.ptr(d_rho), dev.ptr(d_te), dev.ptr(d_b), cells, ctypes.byref(m),
                                      dev.ptr(out), 4 if dtype == "float32" else 8, dev.stream_ptr()))
    return r, theta, phi, out


def precompute_coefficient_bricks(snapshot, scaling, nu_hz: float = 230e9,
                                  dtype: Literal["float32", "float64"] = "float32", coeff_model=None,
                                  stride: int = 1) -> BrickGrid:
    """coefficient_bricks.py:119-152 on the GPU; returns the host brick."""
    r, theta, phi, out = precompute_device_coefficients(snapshot, scaling, nu_hz, dtype, coeff_model, stride)
    return BrickGrid(r, theta, phi, out.cpu().numpy(), spin_a=float(snapshot.spin_a))


def precompute_device_brick(snapshot, scaling, nu_hz: float = 230e9, coeff_model=None, stride: int = 1,
                            precisions=("fp32",)) -> DeviceBrick:
    """The precomputed brick packed for the renderer, without a host copy of
    the coefficients (only the grids pass through the host)."""
    r, theta, phi, out = precompute_device_coefficients(snapshot, scaling, nu_hz, "float32", coeff_model, stride)
    return DeviceBrick.from_device_coeffs(r, theta, phi, out, spin_a=float(snapshot.spin_a), precisions=precisions)
