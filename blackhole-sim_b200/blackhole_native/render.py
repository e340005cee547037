"""Fused GRRT renderer: device-resident bricks, views and the persistent launch.

This is the batched form of the reference's brick renderer
(python/blackhole_sim/accelerated_renderer.py:129-158): every pixel of every
view is one ray through camera -> RK2 Kerr geodesic -> midpoint brick gather
-> Stokes RK2 -> optical-depth cutoff, all inside one persistent CUDA kernel.

Per-step semantics that differ from a literal reading of the reference are
deliberate and documented here:

* the ray loop skips out-of-domain samples and keeps S (the reference
  renderer's behaviour, accelerated_renderer.py:116-118), so the image-level
  meaning of invalid_policy='zero' is "a ray with no valid sample is 0";
* the geodesic ends at the optical-depth cutoff (tau >= max_optical_depth):
  steps after it cannot change the Stokes vector, and they are not counted.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field, replace
from typing import Sequence

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .bricks import BrickGrid, horizon_radius, validate_grid

FOV_20M_AT_1000M = 2.0 * math.degrees(math.atan(20.0 / 1000.0))  # +-20 M field of view at r_obs = 1000 M
EPS_THETA = 1.0e-7


@dataclass(frozen=True)
class View:
    """One pinhole camera view (kerr.py:155-185 LocalCamera +
    accelerated_renderer.py:36-46 AcceleratedRenderConfig)."""

    width: int
    height: int
    spin_a: float = 0.9375
    r_obs: float = 1000.0
    inclination_deg: float = 17.0
    phi_deg: float = 0.0
    fov_y_deg: float = FOV_20M_AT_1000M
    roll_deg: float = 0.0
    max_steps: int = 4096
    h_scale: float = 0.02
    h_min: float = 1.0e-3
    h_max: float = 1.0
    escape_radius: float = 220.0
    affine_to_length_cm: float = 1.0
    max_optical_depth: float = 30.0
    crop: tuple[int, int, int, int] | None = None  # (x0, y0, w, h) of the rendered rectangle
    # Off: the reference's semantics.  On: an inbound ray inside both the innermost
    # photon orbit and the brick's inner radius is captured at that step (no
    # emission can follow in exact arithmetic), which stops the fixed h = 0.02 r
    # step from overshooting into the horizon and flinging the ray back out.
    horizon_guard: bool = False

    @property
    def rect(self) -> tuple[int, int, int, int]:
        return self.crop if self.crop is not None else (0, 0, int(self.width), int(self.height))

    @property
    def pixels(self) -> int:
        x0, y0, w, h = self.rect
        return int(w) * int(h)

    def scaled_step(self, factor: float) -> "View":
        """The same view with every step bound multiplied by ``factor``."""
        return replace(self, h_scale=self.h_scale * factor, h_min=self.h_min * factor, h_max=self.h_max * factor)

    def validate(self) -> None:
        """Host-side checks of kerr.py:30-32 and kerr.py:136-151 (the ZAMO tetrad)."""
        if self.width < 1 or self.height < 1:
            raise ValueError("image width and height must be positive")
        x0, y0, w, h = self.rect
        if w < 1 or h < 1 or x0 < 0 or y0 < 0 or x0 + w > self.width or y0 + h > self.height:
            raise ValueError("view crop rectangle must lie inside the image")
        rp = horizon_radius(self.spin_a)
        th = min(max(math.radians(self.inclination_deg), EPS_THETA), math.pi - EPS_THETA)
        if self.r_obs * self.r_obs - 2.0 * self.r_obs + self.spin_a ** 2 <= 0.0 or self.r_obs <= rp:
            raise ValueError("ZAMO tetrad must be outside the outer horizon")
        if abs(math.sin(th)) < EPS_THETA:
            raise ValueError("ZAMO tetrad is ill-conditioned at the coordinate pole")
        if self.max_steps < 0:
            raise ValueError("max_steps must be non-negative")
        if not (self.h_min > 0.0 and self.h_max >= self.h_min):
            raise ValueError("step bounds must satisfy 0 < h_min <= h_max")

    def to_struct(self, out_offset: int) -> _lib.ViewStruct:
        x0, y0, w, h = self.rect
        s = _lib.ViewStruct()
        s.spin_a = float(self.spin_a)
        s.r_obs = float(self.r_obs)
        s.theta_obs = math.radians(self.inclination_deg)
        s.phi_obs = math.radians(self.phi_deg)
        s.fov_y_deg = float(self.fov_y_deg)
        s.roll_deg = float(self.roll_deg)
        s.h_scale, s.h_min, s.h_max = float(self.h_scale), float(self.h_min), float(self.h_max)
        s.escape_radius = float(self.escape_radius)
        s.affine_to_length_cm = float(self.affine_to_length_cm or 1.0)  # accelerated_renderer.py:146
        s.max_optical_depth = float(self.max_optical_depth)
        s.width, s.height = int(self.width), int(self.height)
        s.x0, s.y0, s.crop_w, s.crop_h = int(x0), int(y0), int(w), int(h)
        s.max_steps = int(self.max_steps)
        s.flags = 1 if self.horizon_guard else 0
        s.out_offset = int(out_offset)
        return s


@dataclass(frozen=True)
class RenderConfig:
    """Launch shape of the persistent kernel (see autotune.py).  The defaults
    are the 80-register variant with every block resident (3 blocks of 256
    threads per SM), 4x8 pixel tiles and batch mode: within 0.5 % of the
    autotuner's best shape on B200 for a 1024x1024 image."""

    block_threads: int = 256
    blocks_per_sm: int = 3
    tile_w: int = 4
    tile_h: int = 8
    refill_min: int = 32
    reg_cap: int = 80

    def to_struct(self, precision: int) -> _lib.RenderConfigStruct:
        c = _lib.RenderConfigStruct()
        c.block_threads, c.blocks_per_sm = int(self.block_threads), int(self.blocks_per_sm)
        c.tile_w, c.tile_h, c.refill_min = int(self.tile_w), int(self.tile_h), int(self.refill_min)
        c.precision = int(precision)
        c.reg_cap = int(self.reg_cap)
        return c


PRECISIONS = {"fp32": 0, "fp64": 1}


class DeviceBrick:
    """A coefficient brick resident in HBM: packed records plus grid tables.

    Records are 12-value cells (the 11 COEFF_NAMES channels and a pad): three
    float4 per cell for the FP32 kernel, six double2 for the FP64 kernel.
    """

    def __init__(self, brick: BrickGrid, device: torch.device | None = None, precisions: Sequence[str] = ("fp32",)):
        self._init_grids(brick.r, brick.theta, brick.phi, brick.spin_a, device)
        c = brick.coeffs.astype(np.float32) if brick.coeffs.dtype == np.float16 else brick.coeffs  # exact widening
        coeffs = dev.to_device(c.reshape(-1), self.device)
        for p in precisions:
            self._pack(coeffs, p)

    @classmethod
    def from_npz(cls, path, device: torch.device | None = None, precisions: Sequence[str] = ("fp32",)) -> "DeviceBrick":
        """A brick file (this package's or the reference's CoefficientBrickGrid
        npz) loaded straight into HBM."""
        return cls(BrickGrid.load_npz(path), device=device, precisions=precisions)

    @classmethod
    def from_device_coeffs(cls, r, theta, phi, coeffs: torch.Tensor, spin_a: float = 0.0,
                           precisions: Sequence[str] = ("fp32",)) -> "DeviceBrick":
        """A brick whose [nr][nt][np][11] values already live on the device
        (float32 or float64 tensor), packed without a host copy."""
        grids = [validate_grid(n, g) for n, g in (("r", r), ("theta", theta), ("phi", phi))]
        obj = cls.__new__(cls)
        obj._init_grids(*grids, spin_a, coeffs.device)
        if coeffs.numel() != obj.cells * 11 or coeffs.dtype not in (torch.float32, torch.float64):
            raise ValueError(f"coeffs must contain exactly r*theta*phi*11 float values; expected {obj.cells * 11}")
        flat = coeffs.contiguous().reshape(-1)
        for p in precisions:
            obj._pack(flat, p)
        return obj

    def _init_grids(self, r, theta, phi, spin_a, device) -> None:
        self.device = device or dev.require_cuda()
        self.nr, self.nt, self.np = int(r.size), int(theta.size), int(phi.size)
        self.shape = (self.nr, self.nt, self.np)
        self.spin_a = float(spin_a)
        self.host_grids = (r, theta, phi)
        self.grids = [dev.to_device(g, self.device) for g in self.host_grids]
        L = _lib.lib()
        nbytes = int(L.bhn_brick_tables_bytes(self.nr, self.nt, self.np))
        self.tables = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        _lib.check(L.bhn_brick_build_tables(dev.ptr(self.grids[0]), self.nr, dev.ptr(self.grids[1]), self.nt,
                                            dev.ptr(self.grids[2]), self.np, dev.ptr(self.tables), dev.stream_ptr()))
        self._records: dict[str, torch.Tensor] = {}

    @property
    def cells(self) -> int:
        return self.nr * self.nt * self.np

    def twin(self) -> "DeviceBrick":
        """A brick on the same grids (shared tables) with its own record
        buffers, initialised to this brick's values."""
        obj = DeviceBrick.__new__(DeviceBrick)
        obj.__dict__.update({k: v for k, v in self.__dict__.items() if k != "_records"})
        obj._records = {p: r.clone() for p, r in self._records.items()}
        return obj

    def reload(self, coeffs: torch.Tensor | np.ndarray, staging: torch.Tensor | None = None,
               check_finite: bool = True) -> torch.Tensor:
        """Replace the brick values (same grids) from host memory: one host->device
        copy (asynchronous when ``coeffs`` is pinned) and a repack on the device.

        ``staging`` is an optional reusable device buffer for the raw values;
        the (possibly new) staging buffer is returned.  With ``check_finite``
        the non-finite count is read back (one synchronisation).
        """
        src = torch.from_numpy(np.ascontiguousarray(coeffs)) if isinstance(coeffs, np.ndarray) else coeffs
        src = (src.float() if src.dtype == torch.float16 else src).reshape(-1)  # exact widening
        if src.numel() != self.cells * 11:
            raise ValueError(f"coeffs must contain exactly r*theta*phi*11 values; expected {self.cells * 11}, "
                             f"got {src.numel()}")
        if staging is None or staging.numel() != src.numel() or staging.dtype != src.dtype:
            staging = torch.empty(src.numel(), dtype=src.dtype, device=self.device)
        staging.copy_(src, non_blocking=True)
        for p in list(self._records):
            self._pack(staging, p, check_finite=check_finite)
        return staging

    def _pack(self, coeffs: torch.Tensor, precision: str, check_finite: bool = True) -> None:
        rb = 4 if precision == "fp32" else 8
        cb = coeffs.element_size()
        rec = self._records.get(precision)
        if rec is None:
            rec = torch.empty(self.cells * 12 * rb, dtype=torch.uint8, device=self.device)
        bad = torch.zeros(1, dtype=torch.int32, device=self.device) if check_finite else None
        _lib.check(_lib.lib().bhn_brick_pack(dev.ptr(coeffs), cb, self.cells, dev.ptr(rec), rb, dev.ptr(bad),
                                             dev.stream_ptr()))
        if check_finite and int(bad.item()):
            raise ValueError("coeffs must contain only finite values")
        self._records[precision] = rec

    def records(self, precision: str) -> torch.Tensor:
        if precision not in self._records:
            raise ValueError(f"brick was not packed for {precision}; pass precisions=(..., '{precision}')")
        return self._records[precision]

    def locate(self, points) -> tuple[np.ndarray, np.ndarray]:
        """Cell indices (i_r, i_theta, i_phi, valid) and float weights of the
        fused kernel's locator for (n, 3) points (test hook for exactness)."""
        pts = dev.to_device(np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1)), self.device)
        n = pts.numel() // 3
        idx = torch.empty(4 * n, dtype=torch.int32, device=self.device)
        w = torch.empty(3 * n, dtype=torch.float32, device=self.device)
        _lib.check(_lib.lib().bhn_brick_locate(dev.ptr(self.tables), self.nr, self.nt, self.np, dev.ptr(pts), n,
                                               dev.ptr(idx), dev.ptr(w), dev.stream_ptr()))
        return idx.cpu().numpy().reshape(n, 4), w.cpu().numpy().reshape(n, 3)


@dataclass
class RenderStats:
    ray_steps: int
    brick_steps: int
    rays: int
    status: dict[str, int]
    queue_fetches: int
    max_h_drift: float
    error_flags: int
    max_h_drift_escaped: float

    @classmethod
    def from_device(cls, t: torch.Tensor) -> "RenderStats":
        raw = bytes(t.cpu().numpy().tobytes())
        s = _lib.RenderStatsStruct.from_buffer_copy(raw)
        return cls(int(s.ray_steps), int(s.brick_steps), int(s.rays),
                   {name: int(s.status[i]) for i, name in enumerate(_lib.RAY_STATUS)}, int(s.queue_fetches),
                   float(s.max_h_drift), int(s.error_flags), float(s.max_h_drift_escaped))


@dataclass
class RenderResult:
    views: list[View]
    out: torch.Tensor                      # (total_pixels, 4) float32 or float64
    offsets: list[int]
    stats_buf: torch.Tensor
    steps: torch.Tensor | None = None
    status: torch.Tensor | None = None
    h_drift: torch.Tensor | None = None
    _stats: RenderStats | None = field(default=None, repr=False)

    def image(self, i: int = 0) -> torch.Tensor:
        v = self.views[i]
        x0, y0, w, h = v.rect
        o = self.offsets[i]
        return self.out[o:o + w * h].view(h, w, 4)

    def per_ray(self, name: str, i: int = 0) -> torch.Tensor | None:
        t = getattr(self, name)
        if t is None:
            return None
        v = self.views[i]
        x0, y0, w, h = v.rect
        o = self.offsets[i]
        return t[o:o + w * h].view(h, w)

    def stats(self) -> RenderStats:
        if self._stats is None:
            self._stats = RenderStats.from_device(self.stats_buf)
        return self._stats


class Renderer:
    """Prepared persistent launch over a fixed list of views.

    ``prepare`` uploads the views and derives their FP64 camera tables on the
    device; ``launch`` (or ``graph_launch`` after ``capture``) then renders all
    views in one kernel.  Output, scratch and statistics buffers are owned here
    and reused by every launch.
    """

    def __init__(self, brick: DeviceBrick, views: Sequence[View], *, config: RenderConfig | None = None,
                 precision: str = "fp32", ray_outputs: bool = False):
        if precision not in PRECISIONS:
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.brick = brick
        self.views = list(views)
        if not self.views:
            raise ValueError("at least one view is required")
        for v in self.views:
            v.validate()
        self.config = config or RenderConfig()
        self.precision = precision
        self.device = brick.device
        L = _lib.lib()
        self.offsets, total = [], 0
        for v in self.views:
            self.offsets.append(total)
            total += v.pixels
        self.total_pixels = total
        odt = torch.float32 if precision == "fp32" else torch.float64
        self.out = torch.zeros((total, 4), dtype=odt, device=self.device)
        self.scratch_bytes = int(L.bhn_render_scratch_bytes(len(self.views)))
        self.scratch = torch.zeros(self.scratch_bytes // 8 + 32, dtype=torch.float64, device=self.device)
        self.stats_buf = torch.zeros(_lib.STATS_BYTES, dtype=torch.uint8, device=self.device)
        self.ray_outputs = ray_outputs
        if ray_outputs:
            self.steps = torch.zeros(total, dtype=torch.int32, device=self.device)
            self.status = torch.zeros(total, dtype=torch.uint8, device=self.device)
            self.h_drift = torch.zeros(total, dtype=torch.float32, device=self.device)
        else:
            self.steps = self.status = self.h_drift = None
        self._graph = None
        self.prepare()

    def _scratch_ptr(self) -> int:
        p = dev.ptr(self.scratch)
        return (p + 255) & ~255

    def _ray_struct(self) -> _lib.RayOutputsStruct:
        r = _lib.RayOutputsStruct()
        r.steps, r.status, r.h_drift = dev.ptr(self.steps), dev.ptr(self.status), dev.ptr(self.h_drift)
        return r

    def prepare(self) -> None:
        arr = (_lib.ViewStruct * len(self.views))(*[v.to_struct(o) for v, o in zip(self.views, self.offsets)])
        self._views_struct = arr
        _lib.check(_lib.lib().bhn_render_prepare(arr, len(self.views), self._scratch_ptr(), self.scratch_bytes,
                                                 dev.stream_ptr()))

    def _args(self):
        b = self.brick
        self._cfg_struct = self.config.to_struct(PRECISIONS[self.precision])
        self._rays_struct = self._ray_struct()
        return (dev.ptr(b.records(self.precision)), dev.ptr(b.tables), b.nr, b.nt, b.np, len(self.views),
                ctypes.byref(self._cfg_struct), dev.ptr(self.out), ctypes.byref(self._rays_struct),
                self._scratch_ptr(), self.scratch_bytes, dev.ptr(self.stats_buf))

    def launch(self) -> RenderResult:
        _lib.check(_lib.lib().bhn_render_launch(*self._args(), dev.stream_ptr()))
        return self.result()

    def capture(self) -> None:
        """Capture the queue reset and the persistent launch into a CUDA graph."""
        self.release_graph()
        g = ctypes.c_void_p()
        _lib.check(_lib.lib().bhn_graph_create(*self._args(), ctypes.byref(g)))
        self._graph = g

    def graph_launch(self) -> RenderResult:
        if self._graph is None:
            self.capture()
        _lib.check(_lib.lib().bhn_graph_launch(self._graph, dev.stream_ptr()))
        return self.result()

    def release_graph(self) -> None:
        if self._graph is not None:
            _lib.lib().bhn_graph_destroy(self._graph)
            self._graph = None

    def __del__(self):
        try:
            self.release_graph()
        except Exception:
            pass

    def result(self) -> RenderResult:
        return RenderResult(self.views, self.out, self.offsets, self.stats_buf, self.steps, self.status, self.h_drift)


class PipelinedRenderer:
    """Renders a sequence of bricks on the same grids (successive snapshots of
    a simulation, say) for fixed views, overlapping data movement with the
    kernel: while brick k renders, brick k + 1 is copied from pinned host memory
    and packed into records on a copy stream and image k - 1 is copied back on
    a third stream.  Two
    record buffers, two raw staging buffers and two compiled launches
    alternate; events order every buffer's reuse.  Host bricks must be pinned
    (``tensor.pin_memory()``) for the copies to overlap."""

    def __init__(self, brick: DeviceBrick, views: Sequence[View], *, config: RenderConfig | None = None,
                 precision: str = "fp32"):
        self.precision = precision
        self.bricks = [brick, brick.twin()]
        self.renderers = [Renderer(b, views, config=config, precision=precision) for b in self.bricks]
        for r in self.renderers:
            r.capture()
        dev_ = brick.device
        self.copy_stream = torch.cuda.Stream(dev_)
        self.d2h_stream = torch.cuda.Stream(dev_)
        self.staging: list[torch.Tensor | None] = [None, None]
        ev = lambda: [torch.cuda.Event(), torch.cuda.Event()]  # noqa: E731
        self.copied, self.packed, self.rendered, self.fetched = ev(), ev(), ev(), ev()
        self.out_shape = self.renderers[0].out.shape
        self.out_dtype = self.renderers[0].out.dtype

    def run(self, host_bricks: Sequence[torch.Tensor], host_outs: Sequence[torch.Tensor]) -> None:
        """Render host_bricks[k] (raw [nr][nt][np][11] values, pinned) into
        host_outs[k % len(host_outs)] (pinned, the renderer's output shape).
        Returns once all work is queued; synchronise the current stream (which
        waits for the copy streams) before reading the last images."""
        compute = torch.cuda.current_stream(self.bricks[0].device)
        cells = self.bricks[0].cells * 11
        # buffers of an earlier run are free once the work queued before this call is done
        self.copy_stream.wait_stream(compute)
        self.d2h_stream.wait_stream(compute)
        for k, hb in enumerate(host_bricks):
            s = k % 2
            src = hb.reshape(-1)
            if src.numel() != cells:
                raise ValueError(f"brick {k} must contain exactly r*theta*phi*11 values; expected {cells}")
            if self.staging[s] is None or self.staging[s].dtype != src.dtype:
                self.staging[s] = torch.empty(cells, dtype=src.dtype, device=self.bricks[0].device)
            with torch.cuda.stream(self.copy_stream):
                # staging[s] and the records of bricks[s] are packed / rendered in
                # stream order here; the records are free once image k - 2 has rendered
                self.staging[s].copy_(src, non_blocking=True)
                self.copied[s].record(self.copy_stream)
                if k >= 2:
                    self.copy_stream.wait_event(self.rendered[s])
                self.bricks[s]._pack(self.staging[s], self.precision, check_finite=False)  # beside render k - 1
                self.packed[s].record(self.copy_stream)
            compute.wait_event(self.packed[s])
            if k >= 2:  # the output buffer is free once image k - 2 has been fetched
                compute.wait_event(self.fetched[s])
            self.renderers[s].graph_launch()
            self.rendered[s].record(compute)
            dst = host_outs[k % len(host_outs)]
            with torch.cuda.stream(self.d2h_stream):
                self.d2h_stream.wait_event(self.rendered[s])
                dst.copy_(self.renderers[s].out, non_blocking=True)
                self.fetched[s].record(self.d2h_stream)
        compute.wait_stream(self.copy_stream)
        compute.wait_stream(self.d2h_stream)

    def release(self) -> None:
        for r in self.renderers:
            r.release_graph()


def render(brick: DeviceBrick, views: Sequence[View] | View, *, precision: str = "fp32",
           config: RenderConfig | None = None, ray_outputs: bool = False) -> RenderResult:
    """Render views of a device brick (device in, device out)."""
    vs = [views] if isinstance(views, View) else list(views)
    return Renderer(brick, vs, config=config, precision=precision, ray_outputs=ray_outputs).launch()


def render_stokes(brick: BrickGrid, views: Sequence[View] | View, *, precision: str = "fp32",
                  config: RenderConfig | None = None) -> list[np.ndarray]:
    """End-to-end form with host buffers: uploads the brick, renders, and returns
    one (h, w, 4) host array of Stokes (I, Q, U, V) per view."""
    db = DeviceBrick(brick, precisions=(precision,))
    res = render(db, views, precision=precision, config=config)
    host = res.out.cpu().numpy()
    out = []
    for v, o in zip(res.views, res.offsets):
        x0, y0, w, h = v.rect
        out.append(host[o:o + w * h].reshape(h, w, 4))
    return out
