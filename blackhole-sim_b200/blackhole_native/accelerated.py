"""The reference's own brick renderer on the GPU.

Drop-in for ``render_stokes_image_bricks`` and ``render_tile_stokes_bricks``
(python/blackhole_sim/accelerated_renderer.py:100-158): per pixel the camera
ray, a fixed-step RK4 Kerr geodesic (kerr.py:306-313, 337-384) and
``integrate_stokes_from_bricks_trace`` -- the coefficient brick sampled at each
segment's midpoint, RK2 or exact Stokes steps, the optical-depth cutoff --
in FP64, one thread per ray (``bhn_brick_trace_render``).  This is the
reference Python's method; ``render`` / ``Renderer`` run the RK2 form with
the step h = 0.02 r in FP32.

The brick follows ``CoefficientBrickGrid`` (coefficient_bricks.py:28-49): its
grids are float32 values, which set the sampled r / theta range.  The
reference interpolates in the brick's dtype with float32 weights (NumPy's
promotion of float32 grids); the GPU does it in float64, so images agree to
float32 rounding.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .grrt import LocalCamera, PolarizedTransferConfig


@dataclass(frozen=True)
class AcceleratedRenderConfig:
    """accelerated_renderer.py:36-46."""

    width: int = 160
    height: int = 90
    camera: LocalCamera = field(default_factory=lambda: LocalCamera.from_degrees(r=55.0, inclination_degrees=65.0,
                                                                                  fov_y_degrees=32.0))
    step: float = 0.06
    max_steps: int = 5000
    escape_radius: float = 220.0
    transfer: PolarizedTransferConfig = field(default_factory=lambda: PolarizedTransferConfig(use_exact_matrix_step=False))
    tile_size: int = 64
    progressive_min_width: int = 480


class BrickTraceConfigStruct(ctypes.Structure):
    """``bhn_brick_trace_config``."""

    _fields_ = [
        ("step", ctypes.c_double),
        ("escape_radius", ctypes.c_double),
        ("length_cm", ctypes.c_double),
        ("max_optical_depth", ctypes.c_double),
        ("max_steps", ctypes.c_int32),
        ("exact_step", ctypes.c_int32),
        ("full_trace", ctypes.c_int32),
        ("coeff_layout", ctypes.c_int32),
    ]


DIAGNOSTICS = ("optical_depth", "sampled_segments", "steps", "status")


def _declare() -> ctypes.CDLL:
    L = _lib.lib()
    fn = L.bhn_brick_trace_render
    vp, i32 = ctypes.c_void_p, ctypes.c_int32
    fn.argtypes = [vp, vp, i32, vp, i32, vp, i32, ctypes.POINTER(_lib.ViewStruct), ctypes.POINTER(BrickTraceConfigStruct),
                   vp, ctypes.c_int64, vp, vp, vp]
    fn.restype = ctypes.c_int
    return L


def _grid(g) -> np.ndarray:
    """A brick axis as CoefficientBrickGrid stores it (float32 values), in float64."""
    a = np.asarray(g, dtype=np.float32).astype(np.float64)
    if a.ndim != 1 or a.size < 2 or np.any(np.diff(a) <= 0.0):
        raise ValueError("brick grids must be strictly increasing 1-D arrays of at least 2 values")
    return np.ascontiguousarray(a)


# bhn_brick_trace_config.coeff_layout
BRICK_F64X11, BRICK_F32X12, BRICK_F64X12 = 0, 1, 2


class DeviceBricks:
    """A ``CoefficientBrickGrid`` checked and uploaded once, for repeated
    renders: float64 grids, and the coefficients as 12-wide cell records (the
    11 channels and a pad, 16-byte aligned) in float32 for a float16 / float32
    brick, else float64 -- the renderer interpolates in float64 either way."""

    def __init__(self, bricks, device: torch.device | None = None):
        coeffs = np.asarray(bricks.coeffs)
        host_grids = [_grid(getattr(bricks, n)) for n in ("r", "theta", "phi")]
        self.shape = tuple(g.size for g in host_grids)
        if coeffs.shape != self.shape + (11,):
            raise ValueError(f"coeffs must have shape {self.shape + (11,)}; got {coeffs.shape}")
        if not torch.cuda.is_available() and not np.all(np.isfinite(coeffs)):
            raise ValueError("coefficient brick contains non-finite values")  # the same error as below, GPU or not
        self.device = device or dev.require_cuda()
        # uploaded in the brick's own dtype, checked and padded to records on the device (widening is exact)
        src = np.ascontiguousarray(coeffs if coeffs.dtype in (np.float16, np.float32, np.float64) else
                                   coeffs.astype(np.float64))
        up = torch.from_numpy(src).to(self.device)
        if not bool(torch.isfinite(up).all()):
            raise ValueError("coefficient brick contains non-finite values")
        self.grids = [torch.as_tensor(g, device=self.device) for g in host_grids]
        wide = torch.float64 if src.dtype == np.float64 else torch.float32
        self.layout = BRICK_F64X12 if wide == torch.float64 else BRICK_F32X12
        self.records = torch.nn.functional.pad(up.to(wide), (0, 1)).contiguous()


def _view_and_config(cfg, snapshot, tile, full_trace=False):
    """The bhn_view (camera, crop) and bhn_brick_trace_config of one call, checked on the host."""
    W, H = int(cfg.width), int(cfg.height)
    if W < 1 or H < 1:
        raise ValueError("image width and height must be positive")
    if not (np.isfinite(cfg.step) and cfg.step > 0.0):
        raise ValueError("step must be finite and positive")
    if int(cfg.max_steps) < 0:
        raise ValueError("max_steps must be non-negative")
    x0, y0, w, h = (0, 0, W, H) if tile is None else (int(tile.x0), int(tile.y0), int(tile.x1 - tile.x0),
                                                       int(tile.y1 - tile.y0))
    if not (0 <= x0 and 0 <= y0 and w >= 0 and h >= 0 and x0 + w <= W and y0 + h <= H):
        raise ValueError(f"tile ({x0}, {y0}, {w}x{h}) lies outside the {W}x{H} image")
    cam = cfg.camera
    v = _lib.ViewStruct()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = float(snapshot.spin_a), float(cam.r), float(cam.theta), float(cam.phi)
    v.fov_y_deg, v.roll_deg = float(cam.fov_y_degrees), float(getattr(cam, "roll_degrees", 0.0))
    v.h_scale, v.h_min, v.h_max = 0.02, 1e-3, 1.0  # unused by the fixed-step loop
    v.escape_radius, v.affine_to_length_cm, v.max_optical_depth = float(cfg.escape_radius), 1.0, 30.0
    v.width, v.height, v.x0, v.y0, v.crop_w, v.crop_h = W, H, x0, y0, w, h
    v.max_steps, v.flags, v.out_offset = int(cfg.max_steps), 0, 0
    t = cfg.transfer
    c = BrickTraceConfigStruct()
    c.step, c.escape_radius = float(cfg.step), float(cfg.escape_radius)
    c.length_cm = float(getattr(t, "affine_to_length_cm", None) or 1.0)  # accelerated_renderer.py:146
    c.max_optical_depth, c.max_steps = float(t.max_optical_depth), int(cfg.max_steps)
    c.exact_step = int(bool(t.use_exact_matrix_step))
    c.full_trace = int(bool(full_trace))
    return v, c, (h, w)


def render_stokes_image_bricks_device(cfg, snapshot, bricks, *, tile=None, diagnostics: bool = False,
                                      device: torch.device | None = None, full_trace: bool = False,
                                      check: bool = True):
    """(h, w, 4) float64 Stokes image of the tile (default: the whole image)
    on the device, and (h, w, 4) diagnostics (columns ``DIAGNOSTICS``) when
    asked.  ``snapshot`` supplies the spin (``spin_a``); ``bricks`` is a
    ``CoefficientBrickGrid``-like object or a ``DeviceBricks``.

    A ray's trace ends where the reference's does (capture, escape radius,
    max_steps, non-finite state), at the optical-depth cutoff, or -- unless
    ``full_trace`` -- once it is past the brick's outer radius moving out with
    no radial turning point ahead (status ``outbound``): nothing after either
    cutoff is sampled, so the image is the same; only the diagnostics' step
    count and status differ from a full trace's.

    ``check`` reads the launch's error word back (a synchronising 4-byte
    copy) and raises if the renderer gave up a wait; unchecked, such a launch
    leaves NaN in the rays it did not finish."""
    # host-side checks first: a bad call fails the same way with or without a GPU
    v, c, (h, w) = _view_and_config(cfg, snapshot, tile, full_trace)
    if not isinstance(bricks, DeviceBricks):
        bricks = DeviceBricks(bricks, device)
    device = bricks.device
    if w == 0 or h == 0:  # an empty tile: the reference's loop over no pixels
        out = torch.zeros((h, w, 4), dtype=torch.float64, device=device)
        return (out, torch.zeros_like(out)) if diagnostics else out
    L = _declare()
    nbytes = int(L.bhn_render_scratch_bytes(1))
    scratch = torch.empty(nbytes // 8 + 64, dtype=torch.float64, device=device)
    sp = (dev.ptr(scratch) + 255) & ~255
    out = torch.empty((h, w, 4), dtype=torch.float64, device=device)
    diag = torch.empty((h, w, 4), dtype=torch.float64, device=device) if diagnostics else None
    g, n = bricks.grids, bricks.shape
    c.coeff_layout = bricks.layout
    _lib.check(L.bhn_brick_trace_render(dev.ptr(bricks.records), dev.ptr(g[0]), n[0], dev.ptr(g[1]), n[1], dev.ptr(g[2]),
                                        n[2], ctypes.byref(v), ctypes.byref(c), sp, nbytes, dev.ptr(out),
                                        dev.ptr(diag), dev.stream_ptr()))
    # word 5 of the scratch (bhn_render_prepare's queue state): bit 0 set when the two-warp form of the
    # renderer gave up a wait between its geodesic and transfer warps (a fault, never a slow image)
    if check and int(scratch.view(torch.int32)[(sp - dev.ptr(scratch)) // 4 + 5].item()) & 1:
        raise RuntimeError("brick renderer: a wait between the geodesic and transfer warps timed out")
    return (out, diag) if diagnostics else out


def render_tile_stokes_bricks(cfg, snapshot, bricks, tile) -> np.ndarray:
    """accelerated_renderer.py:129-150 on the GPU: the (tile.height, tile.width, 4) float64 block."""
    return render_stokes_image_bricks_device(cfg, snapshot, bricks, tile=tile).cpu().numpy()


def render_stokes_image_bricks(cfg, snapshot, bricks) -> np.ndarray:
    """accelerated_renderer.py:153-158 on the GPU: the (H, W, 4) float64 image
    (every pixel in one launch; the reference's tiles change no value)."""
    return render_stokes_image_bricks_device(cfg, snapshot, bricks).cpu().numpy()


@dataclass(frozen=True)
class ProgressiveFrame:
    """accelerated_renderer.py:51-56."""

    level: int
    width: int
    height: int
    stokes: np.ndarray


def render_progressive_stokes_bricks(cfg, snapshot, bricks) -> list[ProgressiveFrame]:
    """accelerated_renderer.py:161-166 on the GPU: one frame per progressive
    level (tiles.progressive_levels), coarsest first; the brick is uploaded once."""
    from dataclasses import replace

    from .tiles import progressive_levels

    db = bricks if isinstance(bricks, DeviceBricks) else None
    frames = []
    for level, w, h in progressive_levels(cfg.width, cfg.height, min_width=cfg.progressive_min_width):
        level_cfg = replace(cfg, width=w, height=h)
        if db is None:  # host-side checks of the first level's call come before the upload
            _view_and_config(level_cfg, snapshot, None)
            db = DeviceBricks(bricks)
        frames.append(ProgressiveFrame(level=level, width=w, height=h,
                                       stokes=render_stokes_image_bricks_device(level_cfg, snapshot, db).cpu().numpy()))
    return frames


def sample_coefficient_brick(bricks, r: float, theta: float, phi: float) -> np.ndarray | None:
    """accelerated_renderer.py:73-97: the 11 coefficients at one point, or None
    outside the brick's nonperiodic r / theta range; through the plugin
    sampler ``sample_brick_trilinear`` (float64 weights on the brick's grid
    values)."""
    from .kernels import sample_brick_trilinear

    grids = [_grid(getattr(bricks, n)) for n in ("r", "theta", "phi")]
    coeffs = np.asarray(bricks.coeffs, dtype=np.float64).ravel()
    out = np.asarray(sample_brick_trilinear(coeffs, *grids, [float(r), float(theta), float(phi)]), dtype=np.float64)
    return None if not np.all(np.isfinite(out)) else out


@dataclass(frozen=True)
class ImageRegressionMetrics:
    """The fields of the reference's ImageRegressionMetrics
    (webgpu_regression.py:27-36) and its default pass thresholds."""

    max_abs: float
    mean_abs: float
    rmse: float
    psnr_db: float
    sha256: str

    @property
    def passed_default(self) -> bool:
        return self.max_abs <= 0.035 and self.mean_abs <= 0.006


def image_metrics(candidate, reference) -> ImageRegressionMetrics:
    """Regression metrics of a candidate image against a reference image, as
    the reference's regression test defines them (webgpu_regression.py:39-48):
    the largest and the mean absolute difference, the RMSE, the PSNR for a
    unit peak (the RMSE floored at 1e-300), and a SHA-256 fingerprint of the
    candidate's float32 bytes.  Host arithmetic on two small images."""
    import hashlib

    cand = np.asarray(candidate, dtype=np.float64)
    ref = np.asarray(reference, dtype=np.float64)
    if cand.shape != ref.shape:
        raise ValueError(f"shape mismatch: {cand.shape} vs {ref.shape}")
    err = np.subtract(cand, ref)
    magnitude = np.abs(err)
    rmse = float(np.sqrt(np.square(err).mean()))
    fingerprint = hashlib.sha256(cand.astype(np.float32).tobytes()).hexdigest()
    return ImageRegressionMetrics(max_abs=float(magnitude.max()), mean_abs=float(magnitude.mean()), rmse=rmse,
                                  psnr_db=float(20.0 * np.log10(1.0 / max(rmse, 1.0e-300))), sha256=fingerprint)


@dataclass(frozen=True)
class SmallRegressionResult:
    """accelerated_renderer.py:59-63."""

    metrics: ImageRegressionMetrics
    reference: np.ndarray
    candidate: np.ndarray


def compare_reference_vs_bricks(reference, candidate) -> SmallRegressionResult:
    """accelerated_renderer.py:169-171: the images' tone-mapped difference."""
    from .grrt import stokes_to_rgb

    metrics = image_metrics(stokes_to_rgb(candidate), stokes_to_rgb(reference))
    return SmallRegressionResult(metrics=metrics, reference=np.asarray(reference), candidate=np.asarray(candidate))


def save_progressive_npz(frame: ProgressiveFrame, path) -> None:
    """accelerated_renderer.py:178-179."""
    from .grrt import save_stokes_npz

    save_stokes_npz(frame.stokes, path)


__all__ = ["AcceleratedRenderConfig", "DIAGNOSTICS", "DeviceBricks", "ImageRegressionMetrics", "ProgressiveFrame",
           "SmallRegressionResult", "compare_reference_vs_bricks", "image_metrics", "render_progressive_stokes_bricks",
           "sample_coefficient_brick", "save_progressive_npz", "render_stokes_image_bricks", "render_stokes_image_bricks_device",
           "render_tile_stokes_bricks"]
