"""Learned step-size proposal for the RK2 ray loop.

Pipeline (all compute in this package's CUDA kernels):

1. ``generate_samples`` runs the step-doubling RK2 controller over seeded
   scenes; every accepted step may be recorded as (8 features at the step
   start, log(h_opt / h_plain)): h_opt = h err^(-1/3) is the step whose
   estimated RK2 error equals the tolerance -- a function of the local state
   only -- and h_plain = clamp(h_scale r, h_min, h_max) the plain step there.
2. ``train`` fits the 8 -> 64 -> 64 -> 1 SiLU network (BF16 weights, FP32
   accumulation) to the standardised log multiplier with the package's
   forward/backward and Adam kernels (minibatch order from a seeded
   permutation).
3. ``render_learned`` runs the ray loop whose step is h_plain times the
   network's multiplier exp(y - margin), floored at ``min_scale``, re-evaluated
   every ``interval`` steps.  With ``check_tol`` > 0 the embedded
   Euler-midpoint difference h |k2 - k1| checks each proposal; a failing
   step is taken by the step-doubling controller (``fallback="controller"``)
   or is the plain step (``fallback="plain"``).  ``brick_scale`` > 0 caps
   steps inside the coefficient brick at that multiple of h_plain, so the
   radiative transfer is resolved as finely as the plain method at
   brick_scale times its step.

The plain fixed-step RK2 method stays the reference: ``render_plain`` and the
FP64 kernel at a finer step measure the learned method's image error.
"""

from __future__ import annotations

import ctypes
import json
import math
from dataclasses import dataclass
from pathlib import Path
from typing import Sequence

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .render import DeviceBrick, RenderConfig, Renderer, View

N_FEATURES = 8
FEATURE_NAMES = ("log_r", "cos_theta", "asinh_p_r", "asinh_p_theta", "spin_a", "log_abs_delta", "p_phi", "log_jI")
# The spin feature is standardised with a fixed scale: training scenes span a
# narrow band of spins and the data spread would magnify any other spin.
FIXED_NORM = {4: (0.5, 0.5)}
FALLBACKS = {"plain": 0, "controller": 1, "retry": 2}
WEIGHTS_DIR = Path(__file__).resolve().parent / "weights"


class AdaptStruct(ctypes.Structure):
    """``bhn_adapt_params``."""

    _fields_ = [
        ("tol", ctypes.c_float),
        ("sample_prob", ctypes.c_float),
        ("h_floor", ctypes.c_float),
        ("h_ceil", ctypes.c_float),
        ("margin", ctypes.c_float),
        ("check_tol", ctypes.c_float),
        ("brick_scale", ctypes.c_float),
        ("min_scale", ctypes.c_float),
        ("interval", ctypes.c_int32),
        ("max_attempts", ctypes.c_int32),
        ("fallback", ctypes.c_int32),
        ("seed", ctypes.c_uint32),
        ("substeps", ctypes.c_int32),
    ]


@dataclass(frozen=True)
class AdaptConfig:
    """Parameters of the step-doubling controller and of the learned loop
    (``bhn_adapt_params``).  The learned loop's defaults are its measured
    operating point on the 2048^2 time-to-image scenes: each proposal taken as
    two RK2 steps of h / 2 under one brick segment (``substeps=2``), proposals
    at exp(-0.6) of the network's h_opt, floored at 0.3 plain steps, the
    Euler-midpoint check at 1e-3 on each half step, and a failing proposal
    retried by its lane with a shorter step (``fallback="retry"``: the plain
    RK2 step again, at most ``max_attempts`` times -- 16, the controller's
    attempt limit too), so every lane of a warp runs the same step; the
    network is evaluated every 32 steps (one evaluation costs about one RK2
    step of the warp; every 16 gave the same images 1-2 % slower, every 64
    fell back more often); in-brick steps are no longer than the plain step."""

    tol: float = 1e-4
    sample_prob: float = 0.0
    h_floor: float = 1e-6
    h_ceil: float = 64.0
    margin: float = 0.6
    check_tol: float = 1e-3
    brick_scale: float = 1.0
    min_scale: float = 0.3
    interval: int = 32
    max_attempts: int = 16
    fallback: str = "retry"        # learned: "retry" -- the lane retries a failing proposal with a shorter
                                   # step next iteration -- or "plain" / "controller" takes that step
    seed: int = 1
    substeps: int = 2              # learned: RK2 steps of h / substeps per brick segment (1 or 2)

    def to_struct(self) -> AdaptStruct:
        if self.fallback not in FALLBACKS:
            raise ValueError(f"fallback must be one of {sorted(FALLBACKS)}")
        s = AdaptStruct()
        s.tol, s.sample_prob, s.h_floor, s.h_ceil = (float(self.tol), float(self.sample_prob), float(self.h_floor),
                                                     float(self.h_ceil))
        s.margin, s.check_tol, s.brick_scale, s.min_scale = (float(self.margin), float(self.check_tol),
                                                             float(self.brick_scale), float(self.min_scale))
        s.interval, s.max_attempts, s.fallback = int(self.interval), int(self.max_attempts), FALLBACKS[self.fallback]
        s.seed = int(self.seed) & 0xFFFFFFFF
        if self.substeps not in (1, 2):
            raise ValueError("substeps must be 1 or 2")
        s.substeps = int(self.substeps)
        return s


def _declare() -> ctypes.CDLL:
    L = _lib.lib()
    if getattr(L, "_learned_declared", False):
        return L
    vp, i64, i32, f = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_float
    cfgp, rayp = ctypes.POINTER(_lib.RenderConfigStruct), ctypes.POINTER(_lib.RayOutputsStruct)
    sig = {
        "bhn_mlp_param_count": ([], i64),
        "bhn_mlp_blob_bytes": ([], i64),
        "bhn_mlp_pack": ([vp, vp, vp, vp], ctypes.c_int),
        "bhn_mlp_grad": ([vp, vp, vp, i64, i64, vp, vp, vp], ctypes.c_int),
        "bhn_mlp_adam": ([vp, vp, vp, vp, f, f, f, f, i32, vp], ctypes.c_int),
        "bhn_mlp_infer": ([vp, vp, i64, vp, vp], ctypes.c_int),
        "bhn_adaptive_launch": ([vp, vp, i32, i32, i32, i32, cfgp, vp, rayp, vp, i64, ctypes.POINTER(AdaptStruct), vp,
                                 vp, ctypes.c_ulonglong, vp, vp], ctypes.c_int),
        "bhn_learned_launch": ([vp, vp, i32, i32, i32, i32, cfgp, vp, rayp, vp, i64, ctypes.POINTER(AdaptStruct), vp,
                                vp, vp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes, fn.restype = args, res
    L._learned_declared = True
    return L


@dataclass
class StepNet:
    """Network parameters (FP32 master copy) and feature standardisation."""

    params: torch.Tensor          # (bhn_mlp_param_count,) float32 on the device
    norm: np.ndarray              # 18 floats: mu_x[8], 1/sigma_x[8], mu_y, sigma_y
    losses: list[float] | None = None
    meta: dict | None = None      # provenance of trained weights (samples, scene seed, tolerance)
    _blob: torch.Tensor | None = None

    @classmethod
    def initial(cls, norm: np.ndarray, seed: int = 0, device=None) -> "StepNet":
        """He-style initialisation (numpy.random.default_rng(seed))."""
        L = _declare()
        n = int(L.bhn_mlp_param_count())
        rng = np.random.default_rng(seed)
        p = np.zeros(n, dtype=np.float32)
        p[0:512] = rng.normal(0, math.sqrt(2.0 / 8), 512)
        p[576:4672] = rng.normal(0, math.sqrt(2.0 / 64), 4096)
        p[4736:4800] = rng.normal(0, math.sqrt(1.0 / 64), 64)
        device = device or dev.require_cuda()
        return cls(torch.from_numpy(p).to(device), np.asarray(norm, dtype=np.float32))

    def blob(self) -> torch.Tensor:
        """The inference blob (BF16 fragments), rebuilt from the parameters."""
        L = _declare()
        if self._blob is None:
            self._blob = torch.empty(int(L.bhn_mlp_blob_bytes()), dtype=torch.uint8, device=self.params.device)
        h_norm = np.ascontiguousarray(self.norm, dtype=np.float32)  # host memory, read before the call returns
        _lib.check(L.bhn_mlp_pack(dev.ptr(self.params), h_norm.ctypes.data, dev.ptr(self._blob), dev.stream_ptr()))
        torch.cuda.current_stream().synchronize()
        return self._blob

    def save(self, path) -> None:
        np.savez_compressed(path, params=self.params.cpu().numpy(), norm=self.norm,
                            losses=np.asarray(self.losses or [], dtype=np.float64),
                            meta=np.asarray(json.dumps(self.meta or {})))

    @classmethod
    def load(cls, path, device=None) -> "StepNet":
        device = device or dev.require_cuda()
        with np.load(path) as z:
            meta = json.loads(str(z["meta"])) if "meta" in z else None
            return cls(torch.from_numpy(z["params"]).to(device), z["norm"].astype(np.float32),
                       [float(x) for x in z["losses"]] if "losses" in z else None, meta)

    def infer(self, features_std: torch.Tensor) -> torch.Tensor:
        """The in-kernel inference path on standardised feature rows (test hook)."""
        L = _declare()
        x = features_std.to(device=self.params.device, dtype=torch.float32).contiguous()
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        _lib.check(L.bhn_mlp_infer(dev.ptr(self.blob()), dev.ptr(x), x.shape[0], dev.ptr(out), dev.stream_ptr()))
        return out


def compute_norm(samples: torch.Tensor) -> np.ndarray:
    """Standardisation of the 8 features and of the log multiplier from the sample rows."""
    s = samples.double()
    mu = s.mean(dim=0).cpu().numpy()
    sd = s.std(dim=0).cpu().numpy()
    sd = np.maximum(sd, 1e-3)
    for k, (m, sc) in FIXED_NORM.items():
        mu[k], sd[k] = m, sc
    norm = np.zeros(18, dtype=np.float32)
    norm[0:8] = mu[0:8]
    norm[8:16] = 1.0 / sd[0:8]
    norm[16], norm[17] = mu[8], sd[8]
    return norm


def standardise(samples: torch.Tensor, norm: np.ndarray) -> torch.Tensor:
    n = torch.from_numpy(norm).to(samples.device)
    out = samples.clone()
    out[:, :8] = (samples[:, :8] - n[0:8]) * n[8:16]
    out[:, 8] = (samples[:, 8] - n[16]) / n[17]
    return out.contiguous()


def _launch_args(rnd: Renderer):
    b = rnd.brick
    rnd._cfg_struct = rnd.config.to_struct(0)
    rnd._rays_struct = rnd._ray_struct()
    return (dev.ptr(b.records("fp32")), dev.ptr(b.tables), b.nr, b.nt, b.np, len(rnd.views),
            ctypes.byref(rnd._cfg_struct), dev.ptr(rnd.out), ctypes.byref(rnd._rays_struct), rnd._scratch_ptr(),
            rnd.scratch_bytes)


@dataclass
class MethodRun:
    renderer: Renderer
    counters: dict
    ms: float

    def image(self, i: int = 0) -> torch.Tensor:
        return self.renderer.result().image(i)


def render_adaptive(brick: DeviceBrick, views: Sequence[View], adapt: AdaptConfig, *, samples: torch.Tensor | None = None,
                    sample_count: torch.Tensor | None = None, config: RenderConfig | None = None,
                    ray_outputs: bool = False, repeats: int = 1) -> MethodRun:
    """Step-doubling controller over the views (optionally recording samples;
    fastest of ``repeats`` launches, which then record samples repeatedly)."""
    L = _declare()
    rnd = Renderer(brick, views, config=config or RenderConfig(256, 4, 4, 8, 32), precision="fp32",
                   ray_outputs=ray_outputs)
    st = adapt.to_struct()
    cap = 0 if samples is None else samples.shape[0]
    best, counters_out = float("inf"), None
    for _ in range(max(1, repeats)):
        counters = torch.zeros(4, dtype=torch.int64, device=brick.device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.check(L.bhn_adaptive_launch(*_launch_args(rnd), ctypes.byref(st), dev.ptr(samples),
                                         dev.ptr(sample_count), cap, dev.ptr(counters), dev.stream_ptr()))
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        if ms < best:
            best = ms
            c = counters.cpu().tolist()
            counters_out = {"rhs_evals": c[0], "steps": c[1], "rejected": c[2]}
    return MethodRun(rnd, counters_out, best)


def render_learned(brick: DeviceBrick, views: Sequence[View], net: StepNet, adapt: AdaptConfig, *,
                   config: RenderConfig | None = None, ray_outputs: bool = False, repeats: int = 1) -> MethodRun:
    """The ray loop with the network's step proposal (fastest of ``repeats`` launches)."""
    L = _declare()
    rnd = Renderer(brick, views, config=config or RenderConfig(128, 5, 4, 8, 32), precision="fp32",
                   ray_outputs=ray_outputs)
    blob = net.blob()
    st = adapt.to_struct()
    best, counters_out = float("inf"), None
    for _ in range(max(1, repeats)):
        counters = torch.zeros(4, dtype=torch.int64, device=brick.device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.check(L.bhn_learned_launch(*_launch_args(rnd), ctypes.byref(st), dev.ptr(blob), dev.ptr(counters),
                                        dev.stream_ptr()))
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        if ms < best:
            best = ms
            c = counters.cpu().tolist()
            counters_out = {"rhs_evals": c[0], "steps": c[1], "fallbacks": c[2], "net_evals_per_warp": c[3]}
    return MethodRun(rnd, counters_out, best)


def render_plain(brick: DeviceBrick, views: Sequence[View], *, precision: str = "fp32",
                 config: RenderConfig | None = None, repeats: int = 1) -> MethodRun:
    """The plain fixed-step method (fastest of ``repeats`` CUDA-graph launches)."""
    rnd = Renderer(brick, views, config=config, precision=precision)
    rnd.capture()
    rnd.graph_launch()
    best = float("inf")
    for _ in range(max(1, repeats)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rnd.graph_launch()
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    st = rnd.result().stats()
    rnd.release_graph()
    return MethodRun(rnd, {"steps": st.ray_steps, "rhs_evals": 2 * st.ray_steps}, best)


def count_samples(brick: DeviceBrick, views: Sequence[View], adapt: AdaptConfig) -> int:
    """How many rows the controller would record with ``adapt`` (a dry run
    into a one-row buffer: the device counter keeps counting past capacity)."""
    row = torch.empty((1, 9), dtype=torch.float32, device=brick.device)
    count = torch.zeros(1, dtype=torch.int64, device=brick.device)
    render_adaptive(brick, views, adapt, samples=row, sample_count=count)
    return int(count.item())


def generate_samples(brick: DeviceBrick, views: Sequence[View], adapt: AdaptConfig, capacity: int) -> torch.Tensor:
    """Run the controller and return the recorded (features, log multiplier) rows."""
    samples = torch.empty((capacity, 9), dtype=torch.float32, device=brick.device)
    count = torch.zeros(1, dtype=torch.int64, device=brick.device)
    render_adaptive(brick, views, adapt, samples=samples, sample_count=count)
    n = min(int(count.item()), capacity)
    return samples[:n].contiguous()


def train(samples: torch.Tensor, *, epochs: int = 6, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          net: StepNet | None = None, log=None) -> StepNet:
    """Fit the network to the standardised log multiplier with the package's kernels."""
    L = _declare()
    device = samples.device
    norm = compute_norm(samples) if net is None else net.norm
    data = standardise(samples, norm)
    net = net or StepNet.initial(norm, seed=seed, device=device)
    n_par = int(L.bhn_mlp_param_count())
    grad = torch.zeros(n_par, dtype=torch.float32, device=device)
    m = torch.zeros_like(grad)
    v = torch.zeros_like(grad)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    n = data.shape[0]
    steps_per_epoch = max(1, n // batch)
    total_steps = epochs * steps_per_epoch
    step = 0
    losses = []
    s = dev.stream_ptr()
    for ep in range(epochs):
        index = torch.randperm(n, generator=gen, device=device)
        loss.zero_()
        for k in range(steps_per_epoch):
            step += 1
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / total_steps))  # cosine decay
            _lib.check(L.bhn_mlp_grad(dev.ptr(net.params), dev.ptr(data), dev.ptr(index), k * batch, batch,
                                      dev.ptr(grad), dev.ptr(loss), s))
            _lib.check(L.bhn_mlp_adam(dev.ptr(net.params), dev.ptr(grad), dev.ptr(m), dev.ptr(v), lr_t, 0.9, 0.999,
                                      1e-8, step, s))
        ep_loss = float(loss.item()) / (steps_per_epoch * batch)
        losses.append(ep_loss)
        if log:
            log(f"epoch {ep}: mse {ep_loss:.5f}")
    net.losses = losses
    net._blob = None
    return net


def shipped_weights() -> StepNet | None:
    """The shipped network (trained on the controller's samples over the seeded 256-view scene), if present."""
    p = WEIGHTS_DIR / "step_net.npz"
    return StepNet.load(p) if p.exists() else None
