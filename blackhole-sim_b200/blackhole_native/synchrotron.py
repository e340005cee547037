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


FRAME_FIELDS = ("n_e_cm3", "theta_e", "b_gauss", "cos_pitch_to_los", "evpa_rad")


@dataclass(frozen=True)
class LocalPlasmaFrame:
    """The plasma quantities a coefficient model reads (the fields of
    synchrotron.py:28-44): electron density [cm^-3], dimensionless electron
    temperature, field strength [G], cosine of the field's pitch to the line
    of sight, and the EVPA the linear terms are rotated by."""

    n_e_cm3: float
    theta_e: float
    b_gauss: float
    cos_pitch_to_los: float = 0.0
    evpa_rad: float = 0.0

    @property
    def b_perp_gauss(self) -> float:
        return abs(self.b_gauss) * float(np.sqrt(max(0.0, 1.0 - self.cos_pitch_to_los ** 2)))

    @property
    def b_parallel_gauss(self) -> float:
        return self.b_gauss * self.cos_pitch_to_los


@dataclass(frozen=True)
class PolarizedCoefficients:
    """The 11 polarized transfer coefficients of one frame, fields named and
    ordered as the reference's PolarizedCoefficients (synchrotron.py:47-64),
    which is the brick's COEFF_NAMES order."""

    j_i: float = 0.0
    j_q: float = 0.0
    j_u: float = 0.0
    j_v: float = 0.0
    alpha_i: float = 0.0
    alpha_q: float = 0.0
    alpha_u: float = 0.0
    alpha_v: float = 0.0
    rho_v: float = 0.0
    rho_q: float = 0.0
    rho_u: float = 0.0

    def as_array(self) -> np.ndarray:
        return np.array([getattr(self, f) for f in self.__dataclass_fields__], dtype=np.float64)

    def as_emission_vector(self) -> np.ndarray:
        return self.as_array()[:4]

    def propagation_matrix(self) -> np.ndarray:
        """K of dS/ds = j - K S: alpha_I on the diagonal, the alphas in the first
        row and column, the rotativities in the symmetric-antisymmetric lower
        block (the matrix of synchrotron.py:82-94)."""
        ai, aq, au, av, rv, rq, ru = self.as_array()[4:]
        k = np.diag([ai, ai, ai, ai])
        k[0, 1:] = k[1:, 0] = (aq, au, av)
        k[1, 2], k[2, 1] = rv, -rv
        k[1, 3], k[3, 1] = -ru, ru
        k[2, 3], k[3, 2] = rq, -rq
        return k


def _frames_array(frames) -> np.ndarray:
    """(n, 5) float64 frames from LocalPlasmaFrame-like objects or an array."""
    if hasattr(frames, "n_e_cm3"):
        frames = [frames]
    if isinstance(frames, (list, tuple)) and frames and hasattr(frames[0], "n_e_cm3"):
        return np.array([[float(getattr(f, k)) for k in FRAME_FIELDS] for f in frames], dtype=np.float64)
    a = np.ascontiguousarray(np.asarray(frames, dtype=np.float64))
    if a.ndim == 1 and a.size == 5:
        a = a.reshape(1, 5)
    if a.ndim != 2 or a.shape[1] != 5:
        raise ValueError("frames must be LocalPlasmaFrame objects or an (n, 5) array of "
                         "(n_e_cm3, theta_e, b_gauss, cos_pitch_to_los, evpa_rad)")
    return a


class _DeviceCoefficients:
    """Per-frame coefficients of a model on the GPU (``bhn_synchrotron_coefficients``)."""

    def coefficients_batch(self, frames, nu_hz: float):
        """(n, 11) coefficients for n frames.  ``frames`` is an (n, 5) array or
        a list of frames (host: a numpy array is returned) or an (n, 5) float64
        CUDA tensor (the result stays on the device)."""
        on_device = isinstance(frames, torch.Tensor) and frames.is_cuda
        if on_device:
            if frames.dtype != torch.float64 or frames.dim() != 2 or frames.shape[1] != 5:
                raise ValueError("device frames must be an (n, 5) float64 tensor")
            fd = frames.contiguous()
        else:
            fd = dev.to_device(_frames_array(frames), dev.require_cuda())
        n = fd.numel() // 5
        if n < 1:
            raise ValueError("at least one plasma frame is required")
        out = torch.empty((n, 11), dtype=torch.float64, device=fd.device)
        m = model_struct(self, nu_hz, _UNIT_SCALING)
        _lib.check(_declare_frames().bhn_synchrotron_coefficients(dev.ptr(fd), n, ctypes.byref(m), dev.ptr(out),
                                                                  dev.stream_ptr()))
        return out if on_device else out.cpu().numpy()

    def coefficients(self, frame, nu_hz: float) -> PolarizedCoefficients:
        """The model's coefficients for one frame (the reference's
        ``coefficients(frame, nu_hz)``), evaluated on the GPU."""
        return PolarizedCoefficients(*self.coefficients_batch([frame], nu_hz)[0].tolist())


@dataclass(frozen=True)
class ThermalSynchrotronCoefficients(_DeviceCoefficients):
    """synchrotron.py:240-275 (Maxwell-Juettner electrons)."""

    gamma_grid_size: int = 192
    pitch_nodes: int = 16
    faraday_rotation_scale: float = 1.0
    faraday_conversion_scale: float = 1.0


@dataclass(frozen=True)
class NonthermalPowerLawSynchrotronCoefficients(_DeviceCoefficients):
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
class HybridSynchrotronCoefficients(_DeviceCoefficients):
    """synchrotron.py:314-325: the sum of a thermal and a power-law component."""

    thermal: ThermalSynchrotronCoefficients = field(default_factory=ThermalSynchrotronCoefficients)
    nonthermal: NonthermalPowerLawSynchrotronCoefficients = field(
        default_factory=NonthermalPowerLawSynchrotronCoefficients)


class _UnitScaling:  # the per-frame models read no plasma scaling
    rho_cgs_per_code = 1.0
    b_gauss_per_code = 1.0
    mean_molecular_weight_per_electron = 1.0


_UNIT_SCALING = _UnitScaling()


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


def _declare_frames() -> ctypes.CDLL:
    L = _lib.lib()
    fn = L.bhn_synchrotron_coefficients
    vp = ctypes.c_void_p
    fn.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(ModelStruct), vp, vp]
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


PIPELINE_MIN_CELLS = 1 << 20   # host-to-host calls this large are pipelined in r slabs
PIPELINE_SLABS = 8


def precompute_coefficient_bricks(snapshot, scaling, nu_hz: float = 230e9,
                                  dtype: Literal["float32", "float16", "float64"] = "float32", coeff_model=None,
                                  stride: int = 1) -> BrickGrid:
    """coefficient_bricks.py:119-152 on the GPU; returns the host brick.

    Large snapshots go through in r slabs: while the device computes slab k,
    slab k + 1's fields are staged in pinned memory and uploaded on a copy
    stream and slab k - 1's coefficients come back on another, so the
    transfers hide behind the kernel.  Slabs change no value.

    float16 bricks are computed in float64 and cast on the host, each value
    rounded once as the reference casts its float64 coefficients, then
    nan_to_num(nan=0, posinf=finfo(float16).max, neginf=0)
    (coefficient_bricks.py:147-151)."""
    if dtype not in ("float32", "float16", "float64"):
        raise ValueError("dtype must be 'float32', 'float16' or 'float64'")
    work = "float64" if dtype == "float16" else dtype
    r, theta, phi, rho, theta_e, b_con = _fields(snapshot, stride)
    shape = (r.size, theta.size, phi.size)
    if int(np.prod(shape)) < PIPELINE_MIN_CELLS or r.size < 2 * PIPELINE_SLABS:
        r, theta, phi, out = precompute_device_coefficients(snapshot, scaling, nu_hz, work, coeff_model, stride)
        coeffs = out.cpu().numpy()
    else:
        coeffs = _precompute_pipelined(rho, theta_e, b_con, scaling, nu_hz, work, coeff_model)
    if dtype == "float16":
        with np.errstate(over="ignore"):
            coeffs = coeffs.astype(np.float16)
        coeffs = np.nan_to_num(coeffs, nan=0.0, posinf=np.finfo(np.float16).max, neginf=0.0)
    return BrickGrid(r, theta, phi, coeffs, spin_a=float(snapshot.spin_a), nu_hz=float(nu_hz))


def _precompute_pipelined(rho: np.ndarray, theta_e: np.ndarray, b_con: np.ndarray, scaling, nu_hz: float,
                          dtype: str, coeff_model) -> np.ndarray:
    L = _declare()
    device = dev.require_cuda()
    nr = rho.shape[0]
    plane = int(np.prod(rho.shape[1:]))
    slab = -(-nr // PIPELINE_SLABS)
    cap = slab * plane
    ndt = np.float32 if dtype == "float32" else np.float64
    tdt = torch.float32 if dtype == "float32" else torch.float64
    out_host = np.empty(rho.shape + (11,), dtype=ndt)
    m = model_struct(coeff_model or HybridSynchrotronCoefficients(), nu_hz, scaling)
    f64 = dict(dtype=torch.float64)
    h_in = [[torch.empty(cap, **f64).pin_memory(), torch.empty(cap, **f64).pin_memory(),
             torch.empty(cap * 4, **f64).pin_memory()] for _ in range(2)]
    d_in = [[torch.empty(cap, device=device, **f64), torch.empty(cap, device=device, **f64),
             torch.empty(cap * 4, device=device, **f64)] for _ in range(2)]
    h_out = [torch.empty(cap * 11, dtype=tdt).pin_memory() for _ in range(2)]
    d_out = [torch.empty(cap * 11, dtype=tdt, device=device) for _ in range(2)]
    compute = torch.cuda.current_stream(device)
    up, down = torch.cuda.Stream(device), torch.cuda.Stream(device)
    up.wait_stream(compute)
    down.wait_stream(compute)
    uploaded = [torch.cuda.Event() for _ in range(2)]
    computed = [torch.cuda.Event() for _ in range(2)]
    downloaded = [torch.cuda.Event() for _ in range(2)]
    rflat, tflat, bflat = rho.reshape(nr, -1), theta_e.reshape(nr, -1), b_con.reshape(nr, -1)
    slabs = [(k * slab, min(nr, (k + 1) * slab)) for k in range(PIPELINE_SLABS) if k * slab < nr]

    def finish(k):  # slab k's coefficients are on the host: copy them out of the pinned buffer
        a, b = slabs[k]
        downloaded[k % 2].synchronize()
        out_host[a:b] = h_out[k % 2][: (b - a) * plane * 11].numpy().reshape((b - a,) + rho.shape[1:] + (11,))

    for k, (a, b) in enumerate(slabs):
        j, n = k % 2, (b - a) * plane
        if k >= 2:
            uploaded[j].synchronize()  # slab k - 2's upload has left this pinned buffer
        h_in[j][0][:n].numpy()[:] = rflat[a:b].reshape(-1)
        h_in[j][1][:n].numpy()[:] = tflat[a:b].reshape(-1)
        h_in[j][2][: 4 * n].numpy()[:] = bflat[a:b].reshape(-1)
        with torch.cuda.stream(up):
            if k >= 2:
                up.wait_event(computed[j])  # slab k - 2's kernel has read these device inputs
            for dst, src, cnt in zip(d_in[j], h_in[j], (n, n, 4 * n)):
                dst[:cnt].copy_(src[:cnt], non_blocking=True)
            uploaded[j].record(up)
        compute.wait_event(uploaded[j])
        if k >= 2:
            compute.wait_event(downloaded[j])  # slab k - 2's coefficients have left this device buffer
        _lib.check(L.bhn_brick_precompute(dev.ptr(d_in[j][0]), dev.ptr(d_in[j][1]), dev.ptr(d_in[j][2]), n,
                                          ctypes.byref(m), dev.ptr(d_out[j]), 4 if dtype == "float32" else 8,
                                          compute.cuda_stream))
        computed[j].record(compute)
        if k >= 1:
            finish(k - 1)  # while slab k computes; frees h_out[(k - 1) % 2] for slab k + 1
        with torch.cuda.stream(down):
            down.wait_event(computed[j])
            h_out[j][: 11 * n].copy_(d_out[j][: 11 * n], non_blocking=True)
            downloaded[j].record(down)
    finish(len(slabs) - 1)
    compute.wait_stream(up)
    compute.wait_stream(down)
    return out_host


def precompute_device_brick(snapshot, scaling, nu_hz: float = 230e9, coeff_model=None, stride: int = 1,
                            precisions=("fp32",)) -> DeviceBrick:
    """The precomputed brick packed for the renderer, without a host copy of
    the coefficients (only the grids pass through the host)."""
    r, theta, phi, out = precompute_device_coefficients(snapshot, scaling, nu_hz, "float32", coeff_model, stride)
    return DeviceBrick.from_device_coeffs(r, theta, phi, out, spin_a=float(snapshot.spin_a), precisions=precisions)
