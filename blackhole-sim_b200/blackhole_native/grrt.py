"""Physical polarized GRRT through a GRMHD snapshot on the GPU.

Drop-in for ``polarized_renderer.render_stokes_image`` (python/blackhole_sim/
polarized_renderer.py:31-70): per pixel the camera ray, a fixed-step RK4 Kerr
geodesic (kerr.py:337-384) and ``integrate_polarized_kerr_grrt``
(polarized_transfer.py:83-145) -- snapshot sampled at every segment's
midpoint, invariant redshift, synchrotron coefficients of the plasma frame at
the emitted frequency, exact or RK2 Stokes steps -- in FP64 CUDA
(``bhn_grrt_render``: rounds of a thread-per-ray trace kernel, a
warp-per-segment coefficient kernel and a thread-per-ray transfer kernel).

The configuration, camera, snapshot and scaling arguments are duck-typed: the
reference's own ``PolarizedRenderConfig`` / ``LocalCamera`` /
``GRMHDSnapshot`` / ``PhysicalScaling`` objects work, and so do this module's
mirrors of them (``seeded_snapshot`` makes a synthetic snapshot).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .synchrotron import HybridSynchrotronCoefficients, ModelStruct, model_struct

G_CGS = 6.67430e-8       # calibration.py:19
C_CGS = 2.99792458e10    # calibration.py:18


@dataclass(frozen=True)
class LocalCamera:
    """kerr.py:155-185 (theta, phi in radians)."""

    r: float = 50.0
    theta: float = math.radians(60.0)
    phi: float = 0.0
    fov_y_degrees: float = 35.0
    roll_degrees: float = 0.0

    @classmethod
    def from_degrees(cls, r: float = 50.0, inclination_degrees: float = 60.0, phi_degrees: float = 0.0,
                     fov_y_degrees: float = 35.0, roll_degrees: float = 0.0) -> "LocalCamera":
        return cls(r=r, theta=math.radians(inclination_degrees), phi=math.radians(phi_degrees),
                   fov_y_degrees=fov_y_degrees, roll_degrees=roll_degrees)


@dataclass(frozen=True)
class PolarizedTransferConfig:
    """polarized_transfer.py:22-28."""

    observing_frequency_hz: float = 230.0e9
    affine_to_length_cm: float | None = None
    max_optical_depth: float = 30.0
    min_redshift: float = 1.0e-8
    use_exact_matrix_step: bool = True


@dataclass(frozen=True)
class PolarizedRenderConfig:
    """polarized_renderer.py:21-30 (``workers`` and ``tone_map`` are accepted and unused: the GPU
    renders every pixel in one launch and returns the raw Stokes image)."""

    width: int = 160
    height: int = 90
    camera: LocalCamera = field(default_factory=lambda: LocalCamera.from_degrees(r=55.0, inclination_degrees=65.0,
                                                                                  fov_y_degrees=32.0))
    step: float = 0.06
    max_steps: int = 5000
    escape_radius: float = 220.0
    workers: int = 1
    transfer: PolarizedTransferConfig = field(default_factory=lambda: PolarizedTransferConfig(use_exact_matrix_step=False))
    tone_map: bool = True


@dataclass
class Snapshot:
    """The fields of ``grmhd.GRMHDSnapshot`` (grmhd.py:54-68) the GPU paths read:
    grids, rho, Theta_e, pressure [nr, nt, np] and b^mu, u^mu [nr, nt, np, 4]."""

    r: np.ndarray
    theta: np.ndarray
    phi: np.ndarray
    rho: np.ndarray
    theta_e: np.ndarray
    pressure: np.ndarray
    b_con: np.ndarray
    u_con: np.ndarray
    spin_a: float


@dataclass(frozen=True)
class PhysicalScaling:
    """calibration.py:48-54 (the unit conversions; rg_cm as calibration.py:107-109)."""

    mass_bh_g: float
    distance_cm: float
    rho_cgs_per_code: float
    b_gauss_per_code: float
    ion_to_electron_temperature_ratio: float = 3.0
    mean_molecular_weight_per_electron: float = 1.0
    flux_scale_jy: float = 1.0

    @property
    def rg_cm(self) -> float:
        return G_CGS * self.mass_bh_g / (C_CGS * C_CGS)


def seeded_snapshot(nr: int = 64, nt: int = 32, nphi: int = 64, spin_a: float = 0.9375, seed: int = 0) -> Snapshot:
    """A seeded GRMHD-like snapshot: r geometric from 1.05 r_+ to 40 M, theta
    cell-centred on (0, pi), phi uniform on [0, 2 pi); torus density
    exp(-(r - 8)^2 / 8 - 4 cos^2 theta) with log-normal noise (sigma 0.2),
    Theta_e log-uniform on [1, 60], pressure rho Theta_e, Gaussian b^mu and a
    slowly rotating flow u = (1, 0, 0, 0.5 r^-1.5)."""
    if min(nr, nt, nphi) < 2:
        raise ValueError("snapshot grids need at least 2 points per axis")
    rng = np.random.default_rng(seed)
    r_plus = 1.0 + math.sqrt(max(1.0 - spin_a * spin_a, 0.0))
    r = np.geomspace(1.05 * r_plus, 40.0, nr)
    theta = (np.arange(nt) + 0.5) * math.pi / nt
    phi = np.linspace(0.0, 2.0 * math.pi, nphi, endpoint=False)
    shape = (nr, nt, nphi)
    rho = np.exp(-((r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(theta)[None, :, None] ** 2) \
        * np.exp(rng.normal(0.0, 0.2, shape))
    theta_e = np.exp(rng.uniform(0.0, math.log(60.0), shape))
    b_con = rng.normal(0.0, 1.0, shape + (4,))
    u_con = np.zeros(shape + (4,))
    u_con[..., 0] = 1.0
    u_con[..., 3] = 0.5 * r[:, None, None] ** -1.5
    return Snapshot(r=r, theta=theta, phi=phi, rho=rho, theta_e=theta_e, pressure=rho * theta_e, b_con=b_con,
                    u_con=u_con, spin_a=float(spin_a))


class GrrtConfigStruct(ctypes.Structure):
    """``bhn_grrt_config``."""

    _fields_ = [
        ("step", ctypes.c_double),
        ("escape_radius", ctypes.c_double),
        ("nu_hz", ctypes.c_double),
        ("length_cm", ctypes.c_double),
        ("max_optical_depth", ctypes.c_double),
        ("min_redshift", ctypes.c_double),
        ("flux_scale", ctypes.c_double),
        ("max_steps", ctypes.c_int32),
        ("exact_step", ctypes.c_int32),
        ("full_trace", ctypes.c_int32),
    ]


DIAGNOSTICS = ("optical_depth", "emitting_steps", "valid_steps", "faraday_depth_abs", "redshift_min", "redshift_max",
               "steps", "status")


def _declare() -> ctypes.CDLL:
    L = _lib.lib()
    L.bhn_grrt_scratch_bytes.argtypes = [ctypes.c_int64, ctypes.c_int32]
    L.bhn_grrt_scratch_bytes.restype = ctypes.c_int64
    fn = L.bhn_grrt_render
    vp, i32 = ctypes.c_void_p, ctypes.c_int32
    fn.argtypes = [vp, vp, i32, vp, i32, vp, i32, ctypes.POINTER(_lib.ViewStruct), ctypes.POINTER(ModelStruct),
                   ctypes.POINTER(GrrtConfigStruct), vp, ctypes.c_int64, vp, vp, vp]
    fn.restype = ctypes.c_int
    return L


def snapshot_fields(snapshot) -> np.ndarray:
    """[nr][nt][np][11] float64: rho, Theta_e, pressure, b^mu, u^mu (grmhd.py:55-68)."""
    shape = (np.asarray(snapshot.r).size, np.asarray(snapshot.theta).size, np.asarray(snapshot.phi).size)
    parts = [np.asarray(snapshot.rho, dtype=np.float64)[..., None], np.asarray(snapshot.theta_e, dtype=np.float64)[..., None],
             np.asarray(snapshot.pressure, dtype=np.float64)[..., None], np.asarray(snapshot.b_con, dtype=np.float64),
             np.asarray(snapshot.u_con, dtype=np.float64)]
    f = np.ascontiguousarray(np.concatenate(parts, axis=-1))
    if f.shape != shape + (11,):
        raise ValueError(f"snapshot fields must have shape {shape} (b_con, u_con {shape + (4,)})")
    return f


def _length_cm(transfer, scaling) -> float:
    if getattr(transfer, "affine_to_length_cm", None) is not None:
        return float(transfer.affine_to_length_cm)
    rg = getattr(scaling, "rg_cm", None)
    if rg is None:
        rg = G_CGS * float(scaling.mass_bh_g) / (C_CGS * C_CGS)  # calibration.py:107-109
    return float(rg)


class DeviceSnapshot:
    """A snapshot's grids and [nr][nt][np][11] field records resident on the
    device, for rendering many images of one snapshot without re-uploading."""

    def __init__(self, snapshot, device: torch.device | None = None):
        device = device or dev.require_cuda()
        for name in ("r", "theta", "phi"):
            g = np.asarray(getattr(snapshot, name), dtype=np.float64)
            if g.ndim != 1 or g.size < 2 or np.any(np.diff(g) <= 0.0):
                raise ValueError(f"{name} grid must be a strictly increasing 1-D array")
        self.device = device
        self.spin_a = float(snapshot.spin_a)
        self.grids = [torch.as_tensor(np.ascontiguousarray(np.asarray(getattr(snapshot, n), dtype=np.float64)),
                                      device=device) for n in ("r", "theta", "phi")]
        self.fields = torch.as_tensor(snapshot_fields(snapshot), device=device)

    @property
    def upload_bytes(self) -> int:
        return int(self.fields.numel() * 8 + sum(g.numel() for g in self.grids) * 8)


SEGMENT_BYTES = 188          # per ray and chunk slot: plasma frame, transfer side data, list index, coefficients
SCRATCH_BUDGET = 512 << 20   # default scratch: chunk = budget / (rays * SEGMENT_BYTES) within [16, 256]


def default_chunk(rays: int) -> int:
    return int(min(256, max(16, SCRATCH_BUDGET // max(1, rays * SEGMENT_BYTES))))


def render_stokes_image_device(cfg, snapshot, scaling, *, coeff_model=None, diagnostics: bool = False,
                               device: torch.device | None = None, out: torch.Tensor | None = None,
                               chunk: int | None = None, full_trace: bool = False):
    """(H, W, 4) float64 Stokes image on the device (and (H, W, 8) diagnostics,
    columns ``DIAGNOSTICS``, when asked).  ``snapshot`` is a host snapshot or a
    ``DeviceSnapshot``; ``out`` an optional preallocated (H, W, 4) float64
    device tensor; ``chunk`` the emitting segments listed per ray and round
    (memory against rounds; the image does not depend on it).  Unless
    ``full_trace``, a ray past the snapshot's outer radius moving out with no
    radial turning point ahead ends there (status 5, outbound): no later
    segment lies in the snapshot, so the image is the same and only the
    diagnostics' step count and status differ from a full trace's."""
    L = _declare()
    ds = snapshot if isinstance(snapshot, DeviceSnapshot) else DeviceSnapshot(snapshot, device)
    device = ds.device
    cam = cfg.camera
    v = _lib.ViewStruct()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = ds.spin_a, float(cam.r), float(cam.theta), float(cam.phi)
    v.fov_y_deg, v.roll_deg = float(cam.fov_y_degrees), float(getattr(cam, "roll_degrees", 0.0))
    v.h_scale, v.h_min, v.h_max = 0.02, 1e-3, 1.0  # unused by the fixed-step loop
    v.escape_radius, v.affine_to_length_cm, v.max_optical_depth = float(cfg.escape_radius), 1.0, 30.0
    v.width, v.height, v.x0, v.y0, v.crop_w, v.crop_h = int(cfg.width), int(cfg.height), 0, 0, int(cfg.width), int(cfg.height)
    v.max_steps, v.flags, v.out_offset = int(cfg.max_steps), 0, 0
    if v.width < 1 or v.height < 1:
        raise ValueError("image width and height must be positive")
    t = cfg.transfer
    c = GrrtConfigStruct()
    c.step, c.escape_radius, c.nu_hz = float(cfg.step), float(cfg.escape_radius), float(t.observing_frequency_hz)
    c.length_cm, c.max_optical_depth, c.min_redshift = _length_cm(t, scaling), float(t.max_optical_depth), float(t.min_redshift)
    c.flux_scale = float(getattr(scaling, "flux_scale_jy", 1.0))
    c.max_steps, c.exact_step = int(cfg.max_steps), int(bool(t.use_exact_matrix_step))
    c.full_trace = int(bool(full_trace))
    m = model_struct(coeff_model or HybridSynchrotronCoefficients(), t.observing_frequency_hz, scaling)
    rays = v.width * v.height
    chunk = default_chunk(rays) if chunk is None else int(chunk)
    if chunk < 1:
        raise ValueError("chunk must be positive")
    nbytes = int(L.bhn_grrt_scratch_bytes(rays, chunk))
    scratch = torch.empty(nbytes // 8 + 64, dtype=torch.float64, device=device)
    sp = (dev.ptr(scratch) + 255) & ~255
    if out is None:
        out = torch.empty((v.height, v.width, 4), dtype=torch.float64, device=device)
    elif (tuple(out.shape) != (v.height, v.width, 4) or out.dtype != torch.float64 or out.device != device
          or not out.is_contiguous()):
        raise ValueError("out must be a contiguous (H, W, 4) float64 tensor on the snapshot's device")
    diag = torch.empty((v.height, v.width, 8), dtype=torch.float64, device=device) if diagnostics else None
    g = ds.grids
    _lib.check(L.bhn_grrt_render(dev.ptr(ds.fields), dev.ptr(g[0]), g[0].numel(), dev.ptr(g[1]), g[1].numel(),
                                 dev.ptr(g[2]), g[2].numel(), ctypes.byref(v), ctypes.byref(m), ctypes.byref(c), sp,
                                 nbytes, dev.ptr(out), dev.ptr(diag), dev.stream_ptr()))
    return (out, diag) if diagnostics else out


def render_stokes_image(cfg, snapshot, scaling, progress: bool = False, *, coeff_model=None):
    """polarized_renderer.py:56-70 on the GPU: the (H, W, 4) float64 Stokes image."""
    return render_stokes_image_device(cfg, snapshot, scaling, coeff_model=coeff_model).cpu().numpy()


def _host_image(stokes_img) -> np.ndarray:
    if isinstance(stokes_img, torch.Tensor):
        stokes_img = stokes_img.detach().cpu().numpy()
    return np.asarray(stokes_img, dtype=np.float64)


def stokes_to_rgb(stokes_img, gamma: float = 2.2) -> np.ndarray:
    """polarized_renderer.py:80-95: the diagnostic colour image of an (H, W, 4)
    Stokes image, (H, W, 3) float64 in [0, 1].  Brightness follows I (negative
    I clipped to 0); the linear polarization sqrt(Q^2 + U^2) adds green, the
    signs of Q and V tint red / blue; every channel is divided by the 99.5th
    percentile of all three, compressed as x / (1 + x) and gamma-encoded.
    Host post-processing of a rendered image (device tensors are copied back)."""
    s = _host_image(stokes_img)
    i = np.maximum(s[..., 0], 0.0)
    q, u, v = s[..., 1], s[..., 2], s[..., 3]
    lin = np.sqrt(q * q + u * u)
    rgb = np.stack([i + 0.35 * np.maximum(q, 0.0) + 0.15 * np.maximum(v, 0.0),
                    i + 0.25 * lin,
                    i + 0.35 * np.maximum(-q, 0.0) + 0.15 * np.maximum(-v, 0.0)], axis=-1)
    peak = float(np.percentile(rgb, 99.5)) if np.any(rgb > 0.0) else 1.0
    rgb = rgb / max(peak, 1.0e-300)
    rgb = rgb / (1.0 + rgb)
    return np.clip(rgb, 0.0, 1.0) ** (1.0 / gamma)


def save_stokes_npz(stokes_img, path) -> None:
    """polarized_renderer.py:98-101: the image as float64 under the key
    ``stokes`` in a compressed npz, parent directories created."""
    from pathlib import Path

    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(p, stokes=_host_image(stokes_img))
