"""CPU oracle of the reference's own brick renderer loop (test infrastructure only).

Restates python/blackhole_sim/accelerated_renderer.py:100-158 for one pixel:
kerr.camera_ray_initial_state and trace_kerr_null_geodesic (fixed-step RK4,
oracle/bhoracle.c bho_trace_rk4), then integrate_stokes_from_bricks_trace over
the stored states: the brick sampled at each segment midpoint with the
sampler's bracket and lerp rules (sample_coefficient_brick, :73-97; here in
float64, oracle.sample_brick_trilinear), ds = L max(|d(r, theta, phi)|,
1e-14), an RK2 or exact Stokes step, the optical-depth cutoff and the final
nan_to_num(nan = posinf = neginf = 0).  Only tests import this module.
"""

from __future__ import annotations

import numpy as np

from . import oracle as O
from . import transfer as T
from .grrt import stokes_step_rk2


def trace_pixel_bricks(view, coeffs, rg, tg, pg, step, max_steps, escape_radius, *, length_cm=1.0, exact=False,
                       max_tau=30.0, px=0, py=0):
    """Stokes (4,) and (tau, sampled segments) of one pixel."""
    aspect = view.width / view.height
    ndc_x = 2.0 * (px + 0.5) / view.width - 1.0
    ndc_y = 1.0 - 2.0 * (py + 0.5) / view.height
    y0, pt, pphi = O.camera_ray(view, ndc_x, ndc_y, aspect)
    states, _ = O.trace_rk4(y0, pt, pphi, view.spin_a, step, max_steps, escape_radius)
    Sv = np.zeros(4)
    tau = 0.0
    sampled = 0
    for i in range(1, len(states)):
        prev, cur = states[i - 1], states[i]
        mid = 0.5 * (prev + cur)
        c = O.sample_brick_trilinear(coeffs, rg, tg, pg, np.array([[mid[1], mid[2], mid[3]]]))[0]
        if not np.all(np.isfinite(c)):
            continue  # outside the nonperiodic r / theta range: no sample
        dl = float(np.linalg.norm(cur[1:4] - prev[1:4]))
        ds = max(length_cm * max(dl, 1.0e-14), 0.0)
        Sv = T.stokes_step_exact(Sv, c, ds) if exact else stokes_step_rk2(Sv, c, ds)
        tau += max(c[4], 0.0) * ds
        sampled += 1
        if tau >= max_tau:
            break
    return np.nan_to_num(Sv, nan=0.0, posinf=0.0, neginf=0.0), (tau, sampled)


def outbound_for_good(states, pt, pphi, a, r_edge):
    """Per stored state (n, 6) of a trace: whether the GPU renderer's exit
    test ends the trace there.  With E = -p_t, L = p_phi, the state's own
    2H = g^{mu nu} p_mu p_nu (the integrator's drift from 0) and the conserved
    K = p_theta^2 + (L / sin - a E sin)^2 - 2H a^2 cos^2, the radial motion obeys
    (Delta p_r)^2 = R(r) = (E (r^2 + a^2) - a L)^2 - Delta (K - 2H r^2)
                        = (E^2 + 2H) r^4 - 4H r^3 + c2 r^2 + 2K r + c0,
    c2 = 2 E B - K + 2H a^2, c0 = B^2 - a^2 K, B = a (a E - L).  For r' >= r
    (K >= 0), R(r') >= e r'^4 + c2 r'^2 + c0 with e = E^2 - |2H| (1 + 2 / r),
    and that is >= e r'^4 / 4 when g(u) = 3/4 e u^2 + c2 u + c0 and g'(u) are
    >= 0 at u = r^2.  The test: past r_edge, p_r > 0, e > 0 and the bound.
    Restated from the Kerr radial potential so tests can check the rule
    against full traces."""
    s = np.asarray(states, dtype=np.float64)
    r, th, pr, pth = s[:, 1], np.clip(s[:, 2], 1.0e-7, np.pi - 1.0e-7), s[:, 4], s[:, 5]
    E, L = -pt, pphi
    sn, cs = np.sin(th), np.cos(th)
    w = L / sn - a * E * sn
    u, a2 = r * r, a * a
    dlt = u - 2.0 * r + a2
    sig = u + a2 * cs * cs
    P = E * (u + a2) - a * L
    with np.errstate(divide="ignore", invalid="ignore"):
        h2 = (dlt * pr * pr + (pth * pth + w * w) - P * P / dlt) / sig  # 2H
        K = pth * pth + w * w - h2 * a2 * cs * cs
        e = E * E - np.abs(h2) * (1.0 + 2.0 / r)
    B = a * (a * E - L)
    e2, c2, c0 = 0.75 * e, 2.0 * E * B - K + h2 * a2, B * B - a2 * K
    return ((r > r_edge) & (pr > 0.0) & (E > 0.0) & (K >= 0.0) & (e > 0.0)
            & (2.0 * e2 * u + c2 >= 0.0) & ((e2 * u + c2) * u + c0 >= 0.0))
