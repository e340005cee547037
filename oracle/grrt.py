"""CPU oracle of the physical polarized GRRT ray loop (test infrastructure only).

Restates python/blackhole_sim/polarized_renderer.py:31-70 for one pixel:
kerr.camera_ray_initial_state and trace_kerr_null_geodesic (fixed-step RK4,
oracle/bhoracle.c bho_trace_rk4), then integrate_polarized_kerr_grrt
(polarized_transfer.py:83-145) over the stored states with the snapshot
sampled as grmhd.GRMHDSnapshot.sample (grmhd.py:106-121, the brick sampler's
bracket and lerp rules) and the Hybrid coefficients of oracle/synchrotron.py.
Only tests import this module.
"""

from __future__ import annotations

import math

import numpy as np

from . import oracle as O
from . import synchrotron as S
from . import transfer as T


def sample_fields(fields, rg, tg, pg, r, th, ph):
    """grmhd.py:106-121 on fields [rho, Theta_e, p, b^mu, u^mu]: (valid, 11 values)."""
    if not (rg[0] <= r <= rg[-1] and tg[0] <= th <= tg[-1]) or not np.all(np.isfinite([r, th, ph])):
        return False, None
    f = O.sample_brick_trilinear(fields, rg, tg, pg, np.array([[r, th, ph]]))[0]
    if f[0] <= 0.0 or f[1] <= 0.0 or not np.all(np.isfinite(f[7:11])):
        return False, None
    return True, f


def stokes_step_rk2(Sv, c, ds):
    """polarized_transfer.py:73-80."""
    K = T.propagation_matrix(c)
    j = np.asarray(c[:4], dtype=float)
    k1 = j - K @ Sv
    mid = Sv + 0.5 * ds * k1
    k2 = j - K @ mid
    return Sv + ds * k2


def trace_pixel(view, fields, rg, tg, pg, scaling, nu_hz, step, max_steps, escape_radius, *, length_cm,
                exact=False, max_tau=30.0, min_redshift=1.0e-8, flux_scale=1.0, thermal=S.THERMAL,
                nonthermal=S.NONTHERMAL, px=0, py=0):
    """Stokes (4,) and (tau, emitting, valid) of one pixel."""
    aspect = view.width / view.height
    ndc_x = 2.0 * (px + 0.5) / view.width - 1.0
    ndc_y = 1.0 - 2.0 * (py + 0.5) / view.height
    y0, pt, pphi = O.camera_ray(view, ndc_x, ndc_y, aspect)
    states, _ = O.trace_rk4(y0, pt, pphi, view.spin_a, step, max_steps, escape_radius)
    Sv = np.zeros(4)
    tau = 0.0
    emit = valid = 0
    for i in range(1, len(states)):
        prev, cur = states[i - 1], states[i]
        mid = 0.5 * (prev + cur)
        ok, f = sample_fields(fields, rg, tg, pg, float(mid[1]), float(mid[2]), float(mid[3]))
        if not ok:
            continue
        valid += 1
        p_cov = np.array([pt, mid[4], mid[5], pphi])
        e_emit = -float(p_cov @ f[7:11])
        g = 1.0 / e_emit if (e_emit > 0.0 and math.isfinite(e_emit)) else 0.0
        if g < min_redshift:
            continue
        n_e, te, b, chi = S.cell_frame(f[0], f[1], f[3:7], scaling["rho_cgs_per_code"], scaling["b_gauss_per_code"],
                                       scaling.get("mu_e", 1.0))
        b_vec = f[4:7]
        b_code = float(np.linalg.norm(b_vec))
        cos_los = 0.0
        if b_code > 0.0:
            k = p_cov[1:]
            nk = float(np.linalg.norm(k))
            if nk > 0.0:
                cos_los = float(np.clip(np.dot(b_vec, k) / (b_code * nk), -1.0, 1.0))
        nu_e = nu_hz / g
        c = S.thermal(n_e, te, b, chi, nu_e, thermal, cos_los) + S.nonthermal(n_e, te, b, chi, nu_e, nonthermal, cos_los)
        c = np.asarray(c, dtype=float)
        c[:4] *= g * g * flux_scale
        c[4:] *= 1.0 / max(g, 1.0e-300)
        dl = float(np.linalg.norm(cur[1:4] - prev[1:4]))
        ds = length_cm * max(e_emit, 0.0) * max(dl, 1.0e-14)
        Sv = T.stokes_step_exact(Sv, c, ds) if exact else stokes_step_rk2(Sv, c, ds)
        tau += max(c[4], 0.0) * ds
        emit += 1
        if tau >= max_tau:
            break
    return Sv, (tau, emit, valid)
