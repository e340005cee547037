"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where a copy of the reference project is readable, naming its python/
directory (or setting BHN_REFERENCE_PYTHON to it):

    python tests/golden/make_golden.py --reference <reference project>/python

Every output value in the fixtures is computed by the reference's own Python
functions (python/blackhole_sim/native_kernels.py, kerr.py,
accelerated_renderer.py, coefficient_bricks.py with synchrotron.py,
polarized_transfer.py, polarized_renderer.py).  The ray-loop fixtures compose those functions the
way the brick renderer does (accelerated_renderer.py:129-150), with the RK2
midpoint step of native/cuda/kerr_stokes_kernel.cu:13 in place of rk4_step and
the variable step h = clamp(0.02 r, 1e-3, 1).  Inputs are seeded and stored
beside the outputs, so the tests never need the reference at run time.
"""

from __future__ import annotations

import argparse
import math
import os
import sys
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _linear_coeff_fixture(nphi: int = 2):
    """The reference test fixture (python/tests/test_native_sampler_parity.py:22-35)."""
    r_grid = np.array([0.0, 1.0])
    theta_grid = np.array([0.0, 1.0])
    phi_grid = np.array([0.0, 1.0]) if nphi == 2 else np.linspace(0.0, 2.0 * math.pi, nphi, endpoint=False)
    coeffs = np.empty((2, 2, nphi, 11))
    for ir in range(2):
        for it in range(2):
            for ip in range(nphi):
                coeffs[ir, it, ip] = 100.0 * ir + 10.0 * it + ip + np.arange(11) * 0.125
    return coeffs, r_grid, theta_grid, phi_grid


def micro_kernels(nk, bench) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(20260101)

    # (1) the reference test fixture with nphi=4 and edge points
    c4, rg, tg, pg = _linear_coeff_fixture(4)
    pts = np.array([
        [0.25, 0.50, math.pi / 4.0],
        [0.50, 0.25, 2.0 * math.pi + math.pi / 4.0],
        [-0.10, 0.50, math.pi / 4.0],
        [0.50, 1.10, math.pi / 4.0],
        [1.00, 1.00, 0.0],                 # last knot in r and theta
        [0.00, 0.00, -1.0e-3],             # first knot, negative phi
        [0.50, 0.50, 3.0 * math.pi / 2.0], # exactly on a phi knot
        [0.50, 0.50, 1.99 * math.pi],      # inside the wrap segment
        [0.50, 0.50, -40.0 * math.pi + 0.3],
        [1.0 + 1e-15, 0.5, 0.5],
    ])
    out["fix4_coeffs"], out["fix4_r"], out["fix4_theta"], out["fix4_phi"], out["fix4_points"] = c4, rg, tg, pg, pts
    out["fix4_sample"] = nk.sample_brick_trilinear_reference(c4, rg, tg, pg, pts)
    out["fix4_mask"] = nk.sample_brick_valid_mask(rg, tg, pts)
    ini = np.zeros((pts.shape[0], 4))
    ini[:, 0], ini[:, 1] = 1.0e-2, 1.0e-3
    out["fix4_initial"] = ini
    for pol in ("nan", "initial", "zero"):
        out[f"fix4_step_{pol}"] = nk.sample_and_step_stokes_reference(c4, rg, tg, pg, pts, ds_cm=0.05, initial=ini,
                                                                       invalid_policy=pol)

    # (2) the reference benchmark fixture (benchmark.py:88-104), 8x6x8 brick, 64 points
    coeffs, rg, tg, pg, pts = bench._sampler_fixture(8, 6, 8, 64)
    out["bench_coeffs"], out["bench_r"], out["bench_theta"], out["bench_phi"], out["bench_points"] = coeffs, rg, tg, pg, pts
    out["bench_sample"] = nk.sample_brick_trilinear_reference(coeffs, rg, tg, pg, pts)
    for pol in ("nan", "initial", "zero"):
        out[f"bench_step_{pol}"] = nk.sample_and_step_stokes_reference(coeffs, rg, tg, pg, pts, ds_cm=0.05,
                                                                        initial=np.array([1e-2, 1e-3, 0.0, 0.0]),
                                                                        invalid_policy=pol)

    # (3) random irregular grids with points on knots, outside, and wrapped phi
    nr, nt, nph = 7, 5, 6
    rgr = np.cumsum(rng.uniform(0.1, 1.0, nr)) + 1.0
    tgr = np.cumsum(rng.uniform(0.05, 0.5, nt))
    pgr = np.sort(rng.uniform(0.0, 2.0 * math.pi, nph))
    cr = rng.normal(size=(nr, nt, nph, 11))
    n = 400
    pr = np.empty((n, 3))
    pr[:, 0] = rng.uniform(rgr[0] - 0.3, rgr[-1] + 0.3, n)
    pr[:, 1] = rng.uniform(tgr[0] - 0.1, tgr[-1] + 0.1, n)
    pr[:, 2] = rng.uniform(-30.0, 30.0, n)
    knots = rng.integers(0, n, 120)
    pr[knots[:40], 0] = rgr[rng.integers(0, nr, 40)]
    pr[knots[40:80], 1] = tgr[rng.integers(0, nt, 40)]
    pr[knots[80:], 2] = pgr[rng.integers(0, nph, 40)] + 2.0 * math.pi * rng.integers(-3, 4, 40)
    out["rand_coeffs"], out["rand_r"], out["rand_theta"], out["rand_phi"], out["rand_points"] = cr, rgr, tgr, pgr, pr
    out["rand_sample"] = nk.sample_brick_trilinear_reference(cr, rgr, tgr, pgr, pr)
    out["rand_mask"] = nk.sample_brick_valid_mask(rgr, tgr, pr)
    rini = rng.normal(size=(n, 4))
    out["rand_initial"] = rini
    for pol in ("nan", "initial", "zero"):
        out[f"rand_step_{pol}"] = nk.sample_and_step_stokes_reference(cr, rgr, tgr, pgr, pr, ds_cm=0.37,
                                                                       initial=rini, invalid_policy=pol)

    # (4) Stokes RK2 over a brick (python/tests/test_native_stokes_parity.py:32-41)
    dc = nk.deterministic_stokes_coefficients(4, 3, 5)
    dini = np.zeros(dc.shape[:-1] + (4,))
    dini[..., 0], dini[..., 1] = 1.0e-2, 1.0e-3
    out["det_coeffs"], out["det_initial"] = dc, dini
    out["det_step"] = nk.stokes_rk2_brick_reference(dc, ds_cm=0.05, initial=dini)
    out["det_step_broadcast"] = nk.stokes_rk2_brick_reference(dc, ds_cm=0.3, initial=np.array([0.5, -0.1, 0.2, 0.05]))
    out["rand_rk2_coeffs"] = rng.normal(size=(257, 11))
    out["rand_rk2_initial"] = rng.normal(size=(257, 4))
    out["rand_rk2_step"] = nk.stokes_rk2_brick_reference(out["rand_rk2_coeffs"], ds_cm=0.11,
                                                         initial=out["rand_rk2_initial"])
    return out


def kerr_fixtures(kerr) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(99)
    # camera rays: (r, incl_deg, fov, a, ndc_x, ndc_y, aspect, roll)
    cams = [
        (1000.0, 17.0, 2.0 * math.degrees(math.atan(20.0 / 1000.0)), 0.9375, 0.3, -0.7, 16.0 / 9.0, 0.0),
        (1000.0, 60.0, 2.0 * math.degrees(math.atan(20.0 / 1000.0)), 0.998, -0.9, 0.9, 1.0, 0.0),
        (55.0, 65.0, 32.0, 0.55, 0.1, 0.2, 16.0 / 9.0, 0.0),
        (40.0, 62.0, 30.0, 0.6, 0.1, -0.2, 16.0 / 9.0, 12.0),
        (500.0, 89.0, 5.0, 0.0, -0.01, 0.02, 1.5, 0.0),
    ]
    y0s, pts_, pps = [], [], []
    for r, inc, fov, a, nx, ny, asp, roll in cams:
        cam = kerr.LocalCamera.from_degrees(r=r, inclination_degrees=inc, fov_y_degrees=fov, roll_degrees=roll)
        y0, pt, pp = kerr.camera_ray_initial_state(cam, a, nx, ny, asp)
        y0s.append(y0), pts_.append(pt), pps.append(pp)
    out["cam_params"] = np.array(cams)
    out["cam_y0"], out["cam_pt"], out["cam_pphi"] = np.array(y0s), np.array(pts_), np.array(pps)

    # RHS, Hamiltonian and metric at random states
    n = 64
    st = np.empty((n, 6))
    st[:, 0] = 0.0
    st[:, 1] = rng.uniform(1.5, 900.0, n)
    st[:, 2] = rng.uniform(1e-3, math.pi - 1e-3, n)
    st[:, 3] = rng.uniform(-10, 10, n)
    st[:, 4] = rng.normal(size=n)
    st[:, 5] = rng.normal(size=n) * 5
    st[:4, 2] = [0.0, 1e-9, math.pi, math.pi - 1e-9]   # pole clamps
    aa = rng.uniform(0.0, 0.998, n)
    pt = -rng.uniform(0.5, 1.5, n)
    pp = rng.normal(size=n) * 3
    out["rhs_states"], out["rhs_a"], out["rhs_pt"], out["rhs_pphi"] = st, aa, pt, pp
    out["rhs_out"] = np.array([kerr.kerr_geodesic_rhs(st[i], aa[i], pt[i], pp[i]) for i in range(n)])
    out["ham_out"] = np.array([kerr.hamiltonian_null(st[i], aa[i], pt[i], pp[i]) for i in range(n)])
    out["gcon_out"] = np.array([kerr.kerr_metric_contravariant(st[i, 1], st[i, 2], aa[i]) for i in range(n)])
    out["gcov_out"] = np.array([kerr.kerr_metric_covariant(st[i, 1], st[i, 2], aa[i]) for i in range(n)])
    h = rng.uniform(1e-3, 1.0, n)
    out["rk2_h"] = h
    out["rk2_out"] = np.array([rk2_step(kerr, st[i], h[i], aa[i], pt[i], pp[i]) for i in range(n)])
    return out


def rk2_step(kerr, y, h, a, p_t, p_phi):
    """RK2 midpoint (native/cuda/kerr_stokes_kernel.cu:13) on kerr.kerr_geodesic_rhs,
    theta clamped like kerr.rk4_step (kerr.py:312)."""
    k1 = kerr.kerr_geodesic_rhs(y, a, p_t, p_phi)
    mid = y + 0.5 * h * k1
    k2 = kerr.kerr_geodesic_rhs(mid, a, p_t, p_phi)
    out = y + h * k2
    out[2] = kerr._safe_theta(float(out[2]))
    return out


def trace_rk2(kerr, y0, p_t, p_phi, a, h_scale, h_min, h_max, max_steps, escape_radius):
    """kerr.trace_kerr_null_geodesic (kerr.py:337-384) with the RK2 step and
    h = clamp(h_scale * r, h_min, h_max) evaluated at the start of each step."""
    y = np.asarray(y0, dtype=float).copy()
    r_plus = kerr.horizon_radius(a)
    states = [y.copy()]
    H0 = abs(kerr.hamiltonian_null(y, a, p_t, p_phi))
    max_h_err = 0.0
    status = "max_steps"
    prev_r = float(y[1])
    steps = 0
    for i in range(1, max_steps + 1):
        h = min(max(h_scale * float(y[1]), h_min), h_max)
        try:
            y = rk2_step(kerr, y, h, a, p_t, p_phi)
            steps += 1
            H = abs(kerr.hamiltonian_null(y, a, p_t, p_phi))
        except (FloatingPointError, ValueError, OverflowError):
            status = "invalid"
            break
        if not np.all(np.isfinite(y)):
            status = "invalid"
            break
        max_h_err = max(max_h_err, abs(H - H0))
        states.append(y.copy())
        r = float(y[1])
        if r <= r_plus * (1.0 + 2.0e-4):
            status = "captured"
            break
        if r > escape_radius and r > prev_r:
            status = "escaped"
            break
        prev_r = r
    if len(states) == 0 or not np.allclose(states[-1], y):
        states.append(y.copy())
    return np.vstack(states), status, max_h_err, steps


STATUS_CODES = {"max_steps": 0, "captured": 1, "escaped": 2, "invalid": 3}


def render_reference(kerr, acc, view: dict, brick) -> dict[str, np.ndarray]:
    """Per-pixel composition of accelerated_renderer.render_tile_stokes_bricks
    (accelerated_renderer.py:129-150) over the crop rectangle."""
    W, H = view["width"], view["height"]
    cam = kerr.LocalCamera.from_degrees(r=view["r_obs"], inclination_degrees=view["inclination_deg"],
                                        phi_degrees=0.0, fov_y_degrees=view["fov_y_deg"])
    aspect = W / H
    x0, y0, cw, ch = view["crop"]
    img = np.zeros((ch, cw, 4))
    steps = np.zeros((ch, cw), dtype=np.int32)
    status = np.zeros((ch, cw), dtype=np.int32)
    drift = np.zeros((ch, cw))
    bricks = SimpleNamespace(r=brick.r, theta=brick.theta, phi=brick.phi, coeffs=brick.coeffs.astype(np.float64))
    for tj in range(ch):
        j = y0 + tj
        ndc_y = 1.0 - 2.0 * (j + 0.5) / H
        for ti in range(cw):
            i = x0 + ti
            ndc_x = 2.0 * (i + 0.5) / W - 1.0
            yy, pt, pp = kerr.camera_ray_initial_state(cam, view["spin_a"], ndc_x, ndc_y, aspect)
            states, st, herr, n = trace_rk2(kerr, yy, pt, pp, view["spin_a"], view["h_scale"], view["h_min"],
                                            view["h_max"], view["max_steps"], view["escape_radius"])
            img[tj, ti] = acc.integrate_stokes_from_bricks_trace(states, bricks, affine_to_length_cm=1.0,
                                                                 max_optical_depth=30.0)
            steps[tj, ti], status[tj, ti], drift[tj, ti] = n, STATUS_CODES[st], herr
    return {"stokes": img, "steps": steps, "status": status, "h_drift": drift}


RAY_VIEWS = {
    # the CPU-runnable configuration as stated: 32x18, r_obs 1000, 64 steps -> all-zero image
    "c1": dict(width=32, height=18, r_obs=1000.0, inclination_deg=17.0,
               fov_y_deg=2.0 * math.degrees(math.atan(20.0 / 1000.0)), spin_a=0.9375, max_steps=64,
               h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0, crop=(0, 0, 32, 18)),
    # nonzero variant: same geometry, enough steps to reach and cross the brick (central 12x8 crop)
    "c1_long": dict(width=32, height=18, r_obs=1000.0, inclination_deg=17.0,
                    fov_y_deg=2.0 * math.degrees(math.atan(20.0 / 1000.0)), spin_a=0.9375, max_steps=1600,
                    h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0, crop=(10, 5, 12, 8)),
    # the reference renderer's default camera distance (accelerated_renderer.py:40): r_obs 55, 65 deg
    "near": dict(width=16, height=12, r_obs=55.0, inclination_deg=65.0, fov_y_deg=32.0, spin_a=0.9375,
                 max_steps=700, h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0, crop=(0, 0, 16, 12)),
}


def ray_fixtures(kerr, acc, bricks_mod) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    brick = bricks_mod.torus_brick(8, 6, 8, spin_a=0.9375, seed=7, dtype=np.float64)
    out["brick_coeffs"], out["brick_r"], out["brick_theta"], out["brick_phi"] = (brick.coeffs, brick.r,
                                                                                  brick.theta, brick.phi)
    for name, view in RAY_VIEWS.items():
        t0 = time.time()
        res = render_reference(kerr, acc, view, brick)
        for k, v in res.items():
            out[f"{name}_{k}"] = v
        out[f"{name}_view"] = np.array([view["width"], view["height"], view["r_obs"], view["inclination_deg"],
                                        view["fov_y_deg"], view["spin_a"], view["max_steps"], view["h_scale"],
                                        view["h_min"], view["h_max"], view["escape_radius"], *view["crop"]])
        print(f"  {name}: {time.time() - t0:.1f}s  nonzero={np.count_nonzero(res['stokes'][..., 0])}", flush=True)
    return out


def precompute_snapshot(seed: int = 7):
    """Seeded small GRMHD-like snapshot: 5 x 4 x 3 cells over the reference's
    usable range (Thetae 0 .. 200 including the 1e-8 floor and cold cells,
    fields of either sign and a zero-field cell)."""
    rng = np.random.default_rng(seed)
    a = 0.9375
    r_plus = 1.0 + math.sqrt(1.0 - a * a)
    r = np.geomspace(1.05 * r_plus, 40.0, 5)
    theta = (np.arange(4) + 0.5) * math.pi / 4.0
    phi = np.linspace(0.0, 2.0 * math.pi, 3, endpoint=False)
    shape = (r.size, theta.size, phi.size)
    rho = np.exp(-((r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(theta)[None, :, None] ** 2) \
        * np.exp(rng.normal(0.0, 0.3, shape))
    theta_e = np.exp(rng.uniform(np.log(0.05), np.log(200.0), shape))
    theta_e[0, 0, 0] = 0.0            # floored to 1e-8 by the reference
    theta_e[0, 1, 0] = 1.0e-3         # cold: no thermal emission at 230 GHz
    b_con = rng.normal(0.0, 1.0, shape + (4,))
    b_con[1, 1, 1, 1:] = 0.0          # zero field: every coefficient 0
    u_con = np.zeros(shape + (4,))
    u_con[..., 0] = 1.0
    pressure = rho * theta_e
    return dict(r=r, theta=theta, phi=phi, rho=rho, theta_e=theta_e, pressure=pressure, b_con=b_con, u_con=u_con,
                spin_a=a)


def precompute_fixtures(grmhd, calibration, cb, synchrotron) -> dict[str, np.ndarray]:
    """precompute_coefficient_bricks (coefficient_bricks.py:119-152) with the
    Hybrid model (synchrotron.py) on the seeded snapshot, in float64 and float32,
    plus the reference's F/G kernel table (synchrotron.py:196-201)."""
    snap = precompute_snapshot()
    scaling = calibration.PhysicalScaling(mass_bh_g=8.54e39, distance_cm=2.57e22, rho_cgs_per_code=3.0e-18,
                                          b_gauss_per_code=25.0)
    g = grmhd.GRMHDSnapshot(**snap)
    out = {f"in_{k}": np.asarray(v) for k, v in snap.items()}
    out["in_rho_cgs_per_code"] = np.asarray(scaling.rho_cgs_per_code)
    out["in_b_gauss_per_code"] = np.asarray(scaling.b_gauss_per_code)
    out["in_mu_e"] = np.asarray(scaling.mean_molecular_weight_per_electron)
    for nu in (230e9, 86e9):
        t0 = time.time()
        b64 = cb.precompute_coefficient_bricks(g, scaling, nu_hz=nu, dtype="float64")
        b32 = cb.precompute_coefficient_bricks(g, scaling, nu_hz=nu, dtype="float32")
        tag = f"{int(nu / 1e9)}"
        out[f"coeffs64_{tag}"] = np.asarray(b64.coeffs)
        out[f"coeffs32_{tag}"] = np.asarray(b32.coeffs)
        print(f"  precompute nu={nu:.3g}: {time.time() - t0:.1f}s", flush=True)
    b2 = cb.precompute_coefficient_bricks(g, scaling, nu_hz=230e9, dtype="float64", stride=2)
    out["coeffs64_230_stride2"] = np.asarray(b2.coeffs)
    xs, F, G = synchrotron._synchrotron_kernel_table()
    out["table_xs"], out["table_F"], out["table_G"] = xs, F, G
    mu, w = np.polynomial.legendre.leggauss(16)
    out["leggauss16_mu"], out["leggauss16_w"] = mu, w
    return out


def frame_fixtures(synchrotron) -> dict[str, np.ndarray]:
    """ThermalSynchrotronCoefficients / NonthermalPowerLawSynchrotronCoefficients /
    HybridSynchrotronCoefficients.coefficients(frame, nu_hz)
    (synchrotron.py:248, 290, 318) on seeded local plasma frames (density,
    temperature, field and pitch spread over the renderer's ranges, plus edge
    frames: no density, no field, a tiny and a zero temperature, field along and
    across the line of sight), four model settings and two frequencies."""
    rng = np.random.default_rng(20261204)
    n = 48
    frames = np.stack([10.0 ** rng.uniform(2, 8, n), 10.0 ** rng.uniform(-1.5, 2.5, n), 10.0 ** rng.uniform(-1, 3, n),
                       rng.uniform(-1, 1, n), rng.uniform(-math.pi, math.pi, n)], axis=1)
    edge = np.array([[0.0, 10.0, 30.0, 0.3, 0.1], [1e6, 10.0, 0.0, 0.3, 0.1], [1e6, 1e-10, 30.0, 0.0, 0.0],
                     [1e6, 0.0, 30.0, 0.5, 1.0], [1e6, 20.0, 30.0, 1.0, -2.0], [1e6, 20.0, 30.0, -1.0, 2.0],
                     [1e6, 20.0, 30.0, 0.0, math.pi / 2], [3e5, 150.0, 500.0, 0.9, -0.7]])
    frames = np.concatenate([frames, edge])
    models = {
        "hybrid": synchrotron.HybridSynchrotronCoefficients(),
        "thermal": synchrotron.ThermalSynchrotronCoefficients(gamma_grid_size=96, pitch_nodes=9,
                                                             faraday_rotation_scale=0.7, faraday_conversion_scale=1.3),
        "nonthermal": synchrotron.NonthermalPowerLawSynchrotronCoefficients(p=2.8, gamma_min=30.0, gamma_max=3e4,
                                                                           nonthermal_fraction=0.1, gamma_grid_size=100,
                                                                           pitch_nodes=12, absorption_scale=0.5,
                                                                           faraday_scale=0.3),
        "hybrid_custom": synchrotron.HybridSynchrotronCoefficients(
            thermal=synchrotron.ThermalSynchrotronCoefficients(gamma_grid_size=64, pitch_nodes=8),
            nonthermal=synchrotron.NonthermalPowerLawSynchrotronCoefficients(gamma_grid_size=300, pitch_nodes=20)),
    }
    out = {"frames": frames}
    for name, model in models.items():
        for nu in (230e9, 86e9):
            t0 = time.time()
            vals = []
            for f in frames:
                frame = synchrotron.LocalPlasmaFrame(*[float(x) for x in f])
                c = model.coefficients(frame, nu)
                vals.append([c.j_i, c.j_q, c.j_u, c.j_v, c.alpha_i, c.alpha_q, c.alpha_u, c.alpha_v, c.rho_v, c.rho_q,
                             c.rho_u])
            out[f"{name}_{int(nu / 1e9)}"] = np.array(vals)
            print(f"  frames {name} nu={nu:.3g}: {time.time() - t0:.1f}s", flush=True)
    return out


def exact_step_fixtures(pt, synchrotron) -> dict[str, np.ndarray]:
    """polarized_transfer.stokes_step_exact (polarized_transfer.py:51-70) on
    seeded coefficient sets and step lengths, including pure emission, pure
    absorption, pure Faraday rotation / conversion, optically thick steps and
    a zero step."""
    rng = np.random.default_rng(20260203)
    cases = []
    for _ in range(40):
        c = rng.normal(0.0, 1.0, 11)
        c[4] = abs(c[4]) + 0.5 * np.linalg.norm(c[5:8])     # alpha_I >= |alpha_pol|: a physical absorber
        cases.append(c)
    special = np.zeros((6, 11))
    special[0, :4] = [1.0, 0.3, -0.2, 0.05]                # emission only
    special[1, 4] = 2.0                                    # absorption only
    special[2, 8:11] = [3.0, 0.0, 0.0]                     # Faraday rotation only
    special[3, 8:11] = [0.0, 1.5, -0.7]                    # Faraday conversion only
    special[4] = [1, 0.5, 0.2, 0.1, 3.0, 1.0, -0.5, 0.3, 5.0, -2.0, 1.0]
    special[5] = [2e-20, 1e-21, 0, 0, 1e-18, 0, 0, 0, 3e-18, 1e-19, 0]
    coeffs = np.vstack([np.array(cases), special])
    ds_list = np.array([0.0, 1.0e-3, 0.1, 1.0, 7.5, 60.0])
    rng2 = np.random.default_rng(5)
    initial = rng2.normal(0.0, 1.0, (coeffs.shape[0], 4))
    out = np.zeros((ds_list.size, coeffs.shape[0], 4))
    for i, ds in enumerate(ds_list):
        for k, c in enumerate(coeffs):
            out[i, k] = pt.stokes_step_exact(initial[k], synchrotron.PolarizedCoefficients(*c), float(ds))
    return {"exact_coeffs": coeffs, "exact_initial": initial, "exact_ds": ds_list, "exact_out": out}


def grrt_snapshot(seed: int = 11):
    """Seeded GRMHD-like snapshot on a 12 x 8 x 6 grid for the physical
    renderer: torus density, Thetae 1..60, random fields, slowly rotating
    flow u = (1, 0, 0, Omega(r))."""
    rng = np.random.default_rng(seed)
    a = 0.9375
    r_plus = 1.0 + math.sqrt(1.0 - a * a)
    r = np.geomspace(1.05 * r_plus, 40.0, 12)
    theta = (np.arange(8) + 0.5) * math.pi / 8.0
    phi = np.linspace(0.0, 2.0 * math.pi, 6, endpoint=False)
    shape = (r.size, theta.size, phi.size)
    rho = np.exp(-((r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(theta)[None, :, None] ** 2) \
        * np.exp(rng.normal(0.0, 0.2, shape))
    theta_e = np.exp(rng.uniform(0.0, np.log(60.0), shape))
    b_con = rng.normal(0.0, 1.0, shape + (4,))
    u_con = np.zeros(shape + (4,))
    u_con[..., 0] = 1.0
    u_con[..., 3] = (0.5 * r[:, None, None] ** -1.5) * np.ones(shape)
    return dict(r=r, theta=theta, phi=phi, rho=rho, theta_e=theta_e, pressure=rho * theta_e, b_con=b_con,
                u_con=u_con, spin_a=a)


def grrt_fixtures(grmhd, calibration, kerr, pr) -> dict[str, np.ndarray]:
    """polarized_renderer.render_stokes_image (polarized_renderer.py:31-70) on a
    4 x 3 image of the seeded snapshot, RK2 and exact Stokes steps."""
    snap = grrt_snapshot()
    g = grmhd.GRMHDSnapshot(**snap)
    scaling = calibration.PhysicalScaling(mass_bh_g=8.54e39, distance_cm=2.57e22, rho_cgs_per_code=3.0e-18,
                                          b_gauss_per_code=25.0)
    out = {f"in_{k}": np.asarray(v) for k, v in snap.items()}
    out["in_rho_cgs_per_code"] = np.asarray(scaling.rho_cgs_per_code)
    out["in_b_gauss_per_code"] = np.asarray(scaling.b_gauss_per_code)
    out["in_rg_cm"] = np.asarray(scaling.rg_cm)
    cam = kerr.LocalCamera.from_degrees(r=30.0, inclination_degrees=65.0, fov_y_degrees=32.0)
    out["cam"] = np.array([cam.r, cam.theta, cam.phi, cam.fov_y_degrees, cam.roll_degrees])
    for exact in (False, True):
        cfg = pr.PolarizedRenderConfig(width=4, height=3, camera=cam, step=0.1, max_steps=900, escape_radius=220.0,
                                       workers=1, transfer=pr.PolarizedTransferConfig(use_exact_matrix_step=exact))
        t0 = time.time()
        out[f"stokes_{'exact' if exact else 'rk2'}"] = pr.render_stokes_image(cfg, g, scaling)
        print(f"  grrt exact={exact}: {time.time() - t0:.1f}s", flush=True)
    return out


def brick_npz_fixture(cb, path) -> None:
    """A small brick written by CoefficientBrickGrid.save_npz (coefficient_bricks.py:57-70)."""
    rng = np.random.default_rng(9)
    r = np.geomspace(1.5, 40.0, 4)
    theta = (np.arange(3) + 0.5) * math.pi / 3.0
    phi = np.linspace(0.0, 2.0 * math.pi, 5, endpoint=False)
    coeffs = rng.uniform(0.0, 1.0, (4, 3, 5, 11)).astype(np.float32)
    cb.CoefficientBrickGrid(r, theta, phi, coeffs, 86e9, 0.5, "float32").save_npz(path)


def rgb_fixtures(pr) -> dict[str, np.ndarray]:
    """polarized_renderer.stokes_to_rgb (polarized_renderer.py:80-95) on a seeded
    Stokes image with negative I, Q and V entries and an all-dark image."""
    rng = np.random.default_rng(12)
    img = rng.normal(0.0, 1.0, (16, 24, 4)) * np.array([1.0, 0.3, 0.3, 0.1])
    img[..., 0] = np.abs(img[..., 0]) * 1e-3
    img[3, 5, 0] = -0.5
    dark = np.zeros((4, 6, 4))
    return {"rgb_in": img, "rgb_out": pr.stokes_to_rgb(img), "rgb_out_g18": pr.stokes_to_rgb(img, gamma=1.8),
            "rgb_dark_in": dark, "rgb_dark_out": pr.stokes_to_rgb(dark)}


def accel_fixtures(cb, acc, kerr, pt, grmhd) -> dict[str, np.ndarray]:
    """accelerated_renderer.render_stokes_image_bricks (accelerated_renderer.py:
    153-158) on a 5 x 4 image of a seeded 10 x 8 x 12 brick, float64 and
    float32 coefficients, RK2 and exact Stokes steps, with a short cutoff run;
    and render_tile_stokes_bricks on one tile."""
    rng = np.random.default_rng(13)
    r = np.geomspace(1.5, 40.0, 10)
    theta = (np.arange(8) + 0.5) * math.pi / 8.0
    phi = np.linspace(0.0, 2.0 * math.pi, 12, endpoint=False)
    dens = np.exp(-((r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(theta)[None, :, None] ** 2) * np.ones((10, 8, 12))
    coeffs = np.zeros((10, 8, 12, 11))
    coeffs[..., :4] = dens[..., None] * np.array([1.0, 0.2, 0.1, 0.02]) * 1e-3
    coeffs[..., 4:8] = 0.1 * coeffs[..., :4] * 10.0
    coeffs[..., 8:] = dens[..., None] * rng.uniform(0.5, 1.5, (10, 8, 12, 3)) * 1e-2
    cam = kerr.LocalCamera.from_degrees(r=30.0, inclination_degrees=70.0, fov_y_degrees=30.0)
    snap = grmhd.GRMHDSnapshot(r=r, theta=theta, phi=phi, rho=dens, theta_e=np.ones_like(dens),
                               pressure=dens, b_con=np.zeros(dens.shape + (4,)), u_con=np.zeros(dens.shape + (4,)),
                               spin_a=0.9375)
    out = {"acc_r": r, "acc_theta": theta, "acc_phi": phi, "acc_coeffs": coeffs, "acc_cam": np.array([cam.r, cam.theta, cam.phi, cam.fov_y_degrees])}
    for dt in ("float64", "float32"):
        bricks = cb.CoefficientBrickGrid(r, theta, phi, coeffs.astype(dt), 230e9, 0.9375, dt)
        for exact in (False, True):
            for max_tau in (30.0, 0.006):
                cfg = acc.AcceleratedRenderConfig(width=5, height=4, camera=cam, step=0.1, max_steps=900,
                                                  transfer=pt.PolarizedTransferConfig(use_exact_matrix_step=exact,
                                                                                      affine_to_length_cm=2.0,
                                                                                      max_optical_depth=max_tau))
                out[f"acc_{dt}_{'exact' if exact else 'rk2'}_{'cut' if max_tau < 1 else 'full'}"] = \
                    acc.render_stokes_image_bricks(cfg, snap, bricks)
        cfg = acc.AcceleratedRenderConfig(width=5, height=4, camera=cam, step=0.1, max_steps=900)
        tile = acc.RenderTile(level=0, y0=1, x0=2, x1=5, y1=3)
        out[f"acc_{dt}_tile"] = acc.render_tile_stokes_bricks(cfg, snap, bricks, tile)
    return out


def accel_regression_fixtures(grmhd, calibration, cb, acc, pr, physics) -> dict[str, np.ndarray]:
    """test_accelerated_renderer.py:17-78 as data: the analytic GRMHD torus
    (generate_analytic_grmhd_torus(0.55, 8, 6, 6)), the Sgr A* scaling at
    Mdot 1e-8, its float32 coefficient brick (precompute_coefficient_bricks),
    the 3 x 2 physical and brick renders with compare_reference_vs_bricks'
    metrics, the progressive frames of an 8 x 6 image and one brick sample."""
    snap = grmhd.generate_analytic_grmhd_torus(spin_a=0.55, nr=8, ntheta=6, nphi=6)
    scaling = calibration.PhysicalScaling.from_mdot(physics.BlackHoleSystem.sgr_a_star(0.55), 1e-8)
    bricks = cb.precompute_coefficient_bricks(snap, scaling, nu_hz=230e9, dtype="float32", stride=1)
    out = {f"snap_{k}": np.asarray(getattr(snap, k)) for k in
           ("r", "theta", "phi", "rho", "theta_e", "pressure", "b_con", "u_con", "spin_a")}
    for k in ("mass_bh_g", "distance_cm", "rho_cgs_per_code", "b_gauss_per_code",
              "ion_to_electron_temperature_ratio", "mean_molecular_weight_per_electron", "flux_scale_jy"):
        out[f"scaling_{k}"] = np.asarray(getattr(scaling, k))
    for k in ("r", "theta", "phi", "coeffs"):
        out[f"brick_{k}"] = np.asarray(getattr(bricks, k))
    ref_cfg = pr.PolarizedRenderConfig(width=3, height=2, max_steps=40, step=0.18, workers=1)
    cand_cfg = acc.AcceleratedRenderConfig(width=3, height=2, max_steps=40, step=0.18, progressive_min_width=2)
    ref = pr.render_stokes_image(ref_cfg, snap, scaling, progress=False)
    cand = acc.render_stokes_image_bricks(cand_cfg, snap, bricks)
    m = acc.compare_reference_vs_bricks(ref, cand).metrics
    out["reg_ref"], out["reg_cand"] = ref, cand
    out["reg_metrics"] = np.array([m.max_abs, m.mean_abs, m.rmse, m.psnr_db])
    frames = acc.render_progressive_stokes_bricks(
        acc.AcceleratedRenderConfig(width=8, height=6, max_steps=30, step=0.2, progressive_min_width=2), snap, bricks)
    out["prog_levels"] = np.array([[f.level, f.width, f.height] for f in frames])
    for i, f in enumerate(frames):
        out[f"prog_{i}"] = f.stokes
    pt = (float(snap.r[3]), float(snap.theta[3]), float(snap.phi[3]))
    out["sample_point"] = np.array(pt)
    out["sample_value"] = acc.sample_coefficient_brick(bricks, *pt)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    env_ref = os.environ.get("BHN_REFERENCE_PYTHON")
    ap.add_argument("--reference", default=env_ref, required=env_ref is None,
                    help="the reference project's python/ directory (default: $BHN_REFERENCE_PYTHON)")
    ap.add_argument("--only", default="",
                    help="comma list of micro,kerr,ray,precompute,exact,grrt,bricknpz,rgb,accel,accelreg,frames")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    sys.path.insert(0, str(REPO / "blackhole-sim_b200"))
    from blackhole_sim import accelerated_renderer as acc, benchmark as bench, kerr, native_kernels as nk
    from blackhole_sim import calibration, grmhd, physics, synchrotron
    from blackhole_sim import polarized_transfer as pt
    from blackhole_sim import polarized_renderer as pr
    from blackhole_sim import coefficient_bricks as cb
    from blackhole_native import bricks as bricks_mod

    only = set(filter(None, args.only.split(",")))
    if not only or "micro" in only:
        np.savez_compressed(HERE / "micro_kernels.npz", **micro_kernels(nk, bench))
        print("wrote micro_kernels.npz")
    if not only or "kerr" in only:
        np.savez_compressed(HERE / "kerr.npz", **kerr_fixtures(kerr))
        print("wrote kerr.npz")
    if not only or "ray" in only:
        np.savez_compressed(HERE / "ray_loop.npz", **ray_fixtures(kerr, acc, bricks_mod))
        print("wrote ray_loop.npz")
    if not only or "precompute" in only:
        np.savez_compressed(HERE / "brick_precompute.npz", **precompute_fixtures(grmhd, calibration, cb, synchrotron))
        print("wrote brick_precompute.npz")
    if not only or "exact" in only:
        np.savez_compressed(HERE / "exact_step.npz", **exact_step_fixtures(pt, synchrotron))
        print("wrote exact_step.npz")
    if not only or "bricknpz" in only:
        brick_npz_fixture(cb, HERE / "reference_brick.npz")
        print("wrote reference_brick.npz")
    if not only or "grrt" in only:
        np.savez_compressed(HERE / "grrt.npz", **grrt_fixtures(grmhd, calibration, kerr, pr))
        print("wrote grrt.npz")
    if not only or "accel" in only:
        np.savez_compressed(HERE / "accel.npz", **accel_fixtures(cb, acc, kerr, pt, grmhd))
        print("wrote accel.npz")
    if not only or "frames" in only:
        np.savez_compressed(HERE / "synchrotron_frames.npz", **frame_fixtures(synchrotron))
        print("wrote synchrotron_frames.npz")
    if not only or "accelreg" in only:
        np.savez_compressed(HERE / "accel_regression.npz",
                            **accel_regression_fixtures(grmhd, calibration, cb, acc, pr, physics))
        print("wrote accel_regression.npz")
    if not only or "rgb" in only:
        np.savez_compressed(HERE / "stokes_rgb.npz", **rgb_fixtures(pr))
        print("wrote stokes_rgb.npz")


if __name__ == "__main__":
    main()
