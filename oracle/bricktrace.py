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
