"""Accuracy studies of the CUDA ray loop, run on the GPU.

* ``precision_study``: 4096 x 4096 rays, a = 0.998, inclination 60 deg,
  max_steps 8192, 256 x 128 x 256 torus brick.  The FP32 kernel (FP64 only in
  the camera set-up, the horizon/turning-point tests and the near-horizon,
  near-pole and extreme-momentum islands) against the FP64 kernel at a 4x
  finer step: Hamiltonian-constraint drift, Stokes I/Q/U/V rel L1 and
  flux-weighted polarization-fraction error.  The FP64 kernel at the same
  step separates rounding from step error.
* ``learned_study``: 2048 x 2048 images of (a = 0.9375, 30 deg) and
  (a = 0.998, 75 deg) through a seed-1 torus brick; time-to-image and Stokes-I
  error of the plain fixed step (h, h/2, h/4, h/8), the step-doubling
  controller and the learned proposal against the FP64 kernel at h/16.
* ``train_shipped``: the network shipped in ``weights/step_net.npz``, trained
  on about 1e7 controller samples over the seeded 256-view scene (uneven view
  sizes, spins U(0, 0.998), inclinations U(5, 85) deg, shared 128 x 64 x 128
  brick; view and brick seed 3, distinct from every evaluation scene).

Error definitions (rel L1 = sum |a - b| / sum |b| over the masked pixels,
as external_validation.py:110-145; m = sqrt(Q^2 + U^2) / I as
polarized_transfer.py:41-44):

* mask: pixels where the FP64 reference is finite, non-negative and stable
  (to 1e-4 relative) under two perturbations: every step bound scaled by
  1 + 1e-6, and the camera distance scaled by 1 + 1e-6 -- the second moves
  every trajectory by about as much as FP32 rounding does, so rays whose
  outcome is decided at rounding level (grazing the spin axis, where the
  method's clamped theta makes the coordinate ds explode) drop out.  The
  precision study's same-step comparison uses the FP64 run at h itself.  In
  the learned study the reference must also be converged (against the FP64
  run at twice its step, to 1e-2 relative).  Every tolerance also carries
  1e-6 (1e-4 for convergence) of the median lit intensity.  Finally the
  reference ray must have kept the null constraint: max |H - H0| <= 1e-2
  (typical rays drift ~1e-4).  A ray past that has stopped being a light ray
  -- the method failed on it (theta clamp at the axis, horizon overshoot), its
  FP64 result is finite garbage (drift up to inf) that is stable under small
  perturbations, and no other precision can be expected to reproduce it.
* capped rel L1: each pixel's |a - b| capped at |b| -- a pixel that blows up
  counts as wholly wrong instead of swamping the sum.
* bad: fraction of masked pixels off by more than 1e-2 relative.

Run as ``python -m blackhole_native.studies {precision,learned,train} --out FILE``.
"""

from __future__ import annotations

import argparse
import json
import time
from dataclasses import replace
from pathlib import Path

import numpy as np
import torch

from . import learned, scenes
from .autotune import cached_config
from .bricks import torus_brick
from .render import DeviceBrick, Renderer, RenderConfig, View


# ------------------------------------------------------------ metrics
def pol_fraction(img: np.ndarray) -> np.ndarray:
    I = np.maximum(img[..., 0], 1e-300)
    with np.errstate(over="ignore", invalid="ignore"):
        return np.sqrt(img[..., 1] ** 2 + img[..., 2] ** 2) / I


def rel_l1(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.abs(b).sum())
    return float(np.abs(a - b).sum() / den) if den > 0 else 0.0


def capped_rel_l1(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.abs(b).sum())
    err = np.minimum(np.nan_to_num(np.abs(a - b), nan=np.inf, posinf=np.inf), np.abs(b))
    return float(err.sum() / den) if den > 0 else 0.0


def flux_weighted_dm(a: np.ndarray, b: np.ndarray, mask: np.ndarray, floor: float = 1e-6) -> float:
    """sum I_b |m_a - m_b| / sum I_b over masked pixels with I_a, I_b above floor x peak I_b."""
    Ib, Ia = b[..., 0], a[..., 0]
    peak = float(Ib[mask].max()) if mask.any() else 0.0
    if peak <= 0:
        return 0.0
    lit = mask & (Ib > floor * peak) & (Ia > floor * peak)
    with np.errstate(over="ignore", invalid="ignore"):
        dm = np.abs(pol_fraction(a) - pol_fraction(b))
    return float(np.sum(Ib[lit] * dm[lit]) / np.sum(Ib[lit])) if lit.any() else 0.0


def median_lit(I: np.ndarray) -> float:
    lit = np.isfinite(I) & (I > 0)
    return float(np.median(I[lit])) if lit.any() else 1.0


def stable_mask(ref: np.ndarray, perts, scale: float) -> np.ndarray:
    """Finite, non-negative pixels of ``ref`` that every perturbed image
    reproduces to 1e-4 relative (plus 1e-6 of ``scale``)."""
    I = ref[..., 0]
    ok = np.isfinite(I) & (I >= 0)
    for pert in perts:
        Ip = pert[..., 0]
        ok &= np.isfinite(Ip) & (np.abs(I - Ip) <= 1e-4 * np.abs(I) + 1e-6 * scale)
    return ok


MAX_DRIFT = 1e-2


def camera_perturbed(view: View) -> View:
    return replace(view, r_obs=view.r_obs * (1.0 + 1e-6))


def image_errors(img: np.ndarray, ref: np.ndarray, mask: np.ndarray, scale: float) -> dict:
    a, b = img.astype(np.float64), ref.astype(np.float64)
    out = {f"rel_l1_{c}": rel_l1(a[..., k][mask], b[..., k][mask]) for k, c in enumerate("IQUV")}
    out["capped_rel_l1_I"] = capped_rel_l1(a[..., 0][mask], b[..., 0][mask])
    d = np.abs(a[..., 0] - b[..., 0])
    out["bad_frac"] = float(np.mean(~(d[mask] <= 1e-2 * np.abs(b[..., 0][mask]) + 1e-4 * scale)))
    out["flux_weighted_dm"] = flux_weighted_dm(a, b, mask)
    return out


# ------------------------------------------------------------ runs
def _render(db: DeviceBrick, view: View, precision: str, config: RenderConfig | None = None,
            ray_outputs: bool = False):
    r = Renderer(db, [view], config=config, precision=precision, ray_outputs=ray_outputs)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    res = r.launch()
    b.record()
    b.synchronize()
    return res, a.elapsed_time(b)


def _drift_summary(drift: np.ndarray, status: np.ndarray) -> dict:
    esc = status == 2
    return {"median": float(np.median(drift)), "p99": float(np.percentile(drift, 99)), "max": float(drift.max()),
            "median_escaped": float(np.median(drift[esc])), "p99_escaped": float(np.percentile(drift[esc], 99)),
            "max_escaped": float(drift[esc].max())}


def precision_study(side: int = 4096, max_steps: int = 8192, log=print) -> dict:
    spin, incl = 0.998, 60.0
    db = DeviceBrick(torus_brick(256, 128, 256, spin_a=spin, seed=0), precisions=("fp32", "fp64"))
    v = View(side, side, spin_a=spin, inclination_deg=incl, max_steps=max_steps, horizon_guard=True)
    v4 = v.scaled_step(0.25)
    cfg = cached_config("image1024", db.device)
    out = {"workload": f"{side}x{side} rays, a={spin}, i={incl} deg, max_steps={max_steps}, 256x128x256x11 float32 "
                       "torus brick (seed 0), RK2 h=0.02 r in [1e-3, 1], horizon guard on",
           "reference": "FP64 kernel at h/4"}
    runs, drifts = {}, {}
    for name, view, prec in (("fp32_h", v, "fp32"), ("fp64_h", v, "fp64"), ("fp64_h_pert", v.scaled_step(1 + 1e-6), "fp64"),
                             ("fp64_h_cam", camera_perturbed(v), "fp64"), ("fp64_h4", v4, "fp64"),
                             ("fp64_h4_pert", v.scaled_step(0.25 * (1 + 1e-6)), "fp64"),
                             ("fp64_h4_cam", camera_perturbed(v4), "fp64")):
        with_rays = name in ("fp32_h", "fp64_h", "fp64_h4")
        res, ms = _render(db, view, prec, config=cfg if prec == "fp32" else None, ray_outputs=with_rays)
        st = res.stats()
        entry = {"ms": ms, "ray_steps": st.ray_steps, "status": st.status}
        if with_rays:
            drift = res.per_ray("h_drift").cpu().numpy().astype(np.float64)
            entry["h_drift"] = _drift_summary(drift, res.per_ray("status").cpu().numpy())
            drifts[name] = drift
        runs[name] = (res.image().cpu().numpy(), entry)
        log(f"{name}: {ms:.1f} ms, {st.ray_steps} ray-steps")
        del res
    ref = runs["fp64_h4"][0]
    scale = median_lit(ref[..., 0])
    mask4 = stable_mask(ref, (runs["fp64_h4_pert"][0], runs["fp64_h4_cam"][0]), scale) & (
        drifts["fp64_h4"] <= MAX_DRIFT)
    # pixels where the method at the step h is itself well conditioned
    mask1 = stable_mask(runs["fp64_h"][0], (runs["fp64_h_pert"][0], runs["fp64_h_cam"][0]),
                        median_lit(runs["fp64_h"][0][..., 0])) & (drifts["fp64_h"] <= MAX_DRIFT)
    out["mask_fraction"] = {"stable_at_h4": float(mask4.mean()), "stable_at_h": float(mask1.mean()),
                            "both": float((mask4 & mask1).mean())}
    out["runs"] = {k: e for k, (_, e) in runs.items()}
    out["errors_vs_fp64_h4"] = {k: image_errors(runs[k][0], ref, mask4, scale) for k in ("fp32_h", "fp64_h")}
    out["errors_vs_fp64_h4_on_both"] = {k: image_errors(runs[k][0], ref, mask4 & mask1, scale)
                                        for k in ("fp32_h", "fp64_h")}
    out["fp32_vs_fp64_same_step"] = image_errors(runs["fp32_h"][0], runs["fp64_h"][0], mask1, scale)
    return out


def fine_step_check(db: DeviceBrick, view: View, crop: tuple[int, int, int, int], fine: int = 4,
                    config: RenderConfig | None = None) -> dict:
    """Stokes error and Hamiltonian drift of the FP32 kernel on a crop of
    ``view`` against the FP64 kernel at 1/``fine`` of the step (with ``fine``
    times the step budget): errors over the pixels whose fine-step FP64 result
    is stable under a 1e-6 step and camera-distance scaling and kept the null
    constraint (|H - H0| <= MAX_DRIFT), plus FP32 against FP64 at the same
    step on the pixels where the method at that step is itself stable.
    ``db`` must hold both record precisions."""
    v = replace(view, crop=crop)
    vf = replace(v.scaled_step(1.0 / fine), max_steps=v.max_steps * fine)
    ref_res = _render(db, vf, "fp64", ray_outputs=True)[0]
    ref = ref_res.image().cpu().numpy()
    ref_drift = ref_res.per_ray("h_drift").cpu().numpy().astype(np.float64)
    del ref_res
    perts = [_render(db, w, "fp64")[0].image().cpu().numpy() for w in (vf.scaled_step(1 + 1e-6), camera_perturbed(vf))]
    scale = median_lit(ref[..., 0])
    mask = stable_mask(ref, perts, scale) & (ref_drift <= MAX_DRIFT)
    r32 = _render(db, v, "fp32", config=config, ray_outputs=True)[0]
    img32 = r32.image().cpu().numpy()
    drift32 = r32.per_ray("h_drift").cpu().numpy().astype(np.float64)
    status32 = r32.per_ray("status").cpu().numpy()
    r64 = _render(db, v, "fp64", ray_outputs=True)[0]
    img64 = r64.image().cpu().numpy()
    drift64 = r64.per_ray("h_drift").cpu().numpy().astype(np.float64)
    p64 = [_render(db, w, "fp64")[0].image().cpu().numpy() for w in (v.scaled_step(1 + 1e-6), camera_perturbed(v))]
    mask1 = stable_mask(img64, p64, median_lit(img64[..., 0])) & (drift64 <= MAX_DRIFT)
    e_fine = image_errors(img32, ref, mask, scale)
    e_same = image_errors(img32, img64, mask1, scale)
    return {"crop": list(crop), "fine_step_factor": 1.0 / fine,
            "mask_fraction": {"fine_step": float(mask.mean()), "same_step": float(mask1.mean())},
            "fp32_vs_fp64_fine": {k: e_fine[k] for k in ("rel_l1_I", "rel_l1_Q", "rel_l1_U", "rel_l1_V",
                                                         "flux_weighted_dm", "bad_frac")},
            "fp32_vs_fp64_same_step": {k: e_same[k] for k in ("rel_l1_I", "flux_weighted_dm", "bad_frac")},
            "h_drift_fp32": _drift_summary(drift32, status32)}


def learned_study(net: learned.StepNet, side: int = 2048, log=print,
                  scenes_=((0.9375, 30.0), (0.998, 75.0))) -> dict:
    cfg = cached_config("image1024", torch.device("cuda"))
    out = {"network": {"features": list(learned.FEATURE_NAMES), "losses": net.losses, "meta": net.meta},
           "scenes": []}
    for spin, incl in scenes_:
        db = DeviceBrick(torus_brick(256, 128, 256, spin_a=spin, seed=1), precisions=("fp32", "fp64"))
        v = View(side, side, spin_a=spin, inclination_deg=incl, max_steps=65536, horizon_guard=True)
        v16 = v.scaled_step(1 / 16)
        ref_res = _render(db, v16, "fp64", ray_outputs=True)[0]
        ref = ref_res.image().cpu().numpy()
        ref_drift = ref_res.per_ray("h_drift").cpu().numpy().astype(np.float64)
        del ref_res
        ref8 = _render(db, v.scaled_step(1 / 8), "fp64")[0].image().cpu().numpy()
        perts = [_render(db, w, "fp64")[0].image().cpu().numpy()
                 for w in (v.scaled_step(1 / 16 * (1 + 1e-6)), camera_perturbed(v16))]
        scale = median_lit(ref[..., 0])
        mask = stable_mask(ref, perts, scale) & np.isfinite(ref8[..., 0]) & (
            np.abs(ref8[..., 0] - ref[..., 0]) <= 1e-2 * np.abs(ref[..., 0]) + 1e-4 * scale) & (ref_drift <= MAX_DRIFT)
        sc = {"spin_a": spin, "inclination_deg": incl, "side": side, "mask_fraction": float(mask.mean()),
              "fp64_h8_vs_h16": image_errors(ref8, ref, mask, scale), "runs": []}
        log(f"scene a={spin} i={incl}: mask {mask.mean():.4f}")

        def record(method, params, run):
            img = run.image().cpu().numpy()
            e = {"method": method, **params, "ms": run.ms, **run.counters, **image_errors(img, ref, mask, scale)}
            sc["runs"].append(e)
            log(f"  {method} {params}: {run.ms:.2f} ms, capped {e['capped_rel_l1_I']:.2e}, rel {e['rel_l1_I']:.2e}, "
                f"bad {e['bad_frac']:.2e}")

        for f in (1.0, 0.5, 0.25, 0.125):
            record("plain", {"step_factor": f}, learned.render_plain(db, [v.scaled_step(f)], config=cfg, repeats=3))
        for bs in (1.0, 0.5, 0.25):
            for tol in (1e-4, 1e-5):
                record("controller", {"tol": tol, "brick_scale": bs},
                       learned.render_adaptive(db, [v], learned.AdaptConfig(tol=tol, brick_scale=bs), repeats=3))
            for fb in ("retry", "controller", "plain"):
                record("learned", {"fallback": fb, "brick_scale": bs},
                       learned.render_learned(db, [v], net, learned.AdaptConfig(brick_scale=bs, fallback=fb), repeats=3))
        best = {}
        for e in sc["runs"]:
            if e["rel_l1_I"] <= 1e-3:
                k = e["method"] if e["method"] != "learned" else f"learned/{e['fallback']}"
                if k not in best or e["ms"] < best[k]["ms"]:
                    best[k] = e
        sc["time_to_image_1e-3"] = {k: {"ms": e["ms"], "rel_l1_I": e["rel_l1_I"]} for k, e in best.items()}
        out["scenes"].append(sc)
    return out


def train_shipped(n_samples: int = 10_000_000, seed: int = 3, epochs: int = 8, log=print) -> learned.StepNet:
    db = DeviceBrick(scenes.shared_brick(seed=seed), precisions=("fp32",))
    views = [replace(vw, horizon_guard=True) for vw in scenes.uneven_views(256, seed=seed)]
    pilot = 1e-3
    count = learned.count_samples(db, views, learned.AdaptConfig(tol=1e-4, sample_prob=pilot, brick_scale=1.0))
    prob = min(1.0, pilot * n_samples / max(count, 1))
    samples = learned.generate_samples(db, views, learned.AdaptConfig(tol=1e-4, sample_prob=prob, brick_scale=1.0),
                                       int(n_samples * 1.2))
    log(f"pilot {count} samples at p={pilot}; {samples.shape[0]} samples at p={prob:.3g}")
    net = learned.train(samples, epochs=epochs, batch=4096, lr=3e-3, seed=0, log=log)
    net.meta = {"samples": int(samples.shape[0]), "sample_prob": prob, "scene_seed": seed, "tol": 1e-4,
                "scene": "256 uneven views (scenes.uneven_views), shared 128x64x128 brick, horizon guard on"}
    return net


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("study", choices=["precision", "learned", "train"])
    ap.add_argument("--out", required=True, help="JSON report (train: the .npz weights)")
    ap.add_argument("--side", type=int, default=0)
    ap.add_argument("--weights", default=None, help="learned: network .npz (default: the shipped weights)")
    args = ap.parse_args()
    t0 = time.time()
    if args.study == "train":
        net = train_shipped()
        net.save(args.out)
        print(json.dumps({"weights": args.out, "losses": net.losses, **net.meta, "seconds": time.time() - t0}))
        return
    if args.study == "precision":
        rep = precision_study(side=args.side or 4096)
    else:
        net = learned.StepNet.load(args.weights) if args.weights else learned.shipped_weights()
        if net is None:
            raise SystemExit("no network weights: train them first (studies train --out ...)")
        rep = learned_study(net, side=args.side or 2048)
    rep["seconds"] = time.time() - t0
    Path(args.out).write_text(json.dumps(rep, indent=1))
    print(json.dumps({"study": args.study, "out": args.out, "seconds": rep["seconds"]}))


if __name__ == "__main__":
    main()
