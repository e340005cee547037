"""The CPU oracle against the golden vectors made by the reference itself.

The micro-kernels and the Kerr geometry must match bit for bit (they are the
same float64 operations in the same order); the composed ray loop to ~1e-12
(only libm / BLAS summation order differs).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden_view, linear_coeff_fixture, rust_linear_fixture

PREFIXES = ("fix4", "bench", "rand")
DS = {"fix4": 0.05, "bench": 0.05, "rand": 0.37}


def _initial(g, pre):
    return g[f"{pre}_initial"] if f"{pre}_initial" in g else np.array([1e-2, 1e-3, 0.0, 0.0])


@pytest.mark.parametrize("pre", PREFIXES)
def test_sampler_bit_exact(micro_golden, pre):
    g = micro_golden
    out = O.sample_brick_trilinear(g[f"{pre}_coeffs"], g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_phi"],
                                   g[f"{pre}_points"])
    assert np.array_equal(out, g[f"{pre}_sample"], equal_nan=True)


@pytest.mark.parametrize("pre", PREFIXES)
@pytest.mark.parametrize("policy", ["nan", "initial", "zero"])
def test_sample_and_step_bit_exact(micro_golden, pre, policy):
    g = micro_golden
    out = O.sample_and_step_stokes(g[f"{pre}_coeffs"], g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_phi"],
                                   g[f"{pre}_points"], DS[pre], _initial(g, pre), policy)
    assert np.array_equal(out, g[f"{pre}_step_{policy}"], equal_nan=True)


def test_valid_mask_bit_exact(micro_golden):
    g = micro_golden
    for pre in ("fix4", "rand"):
        assert np.array_equal(O.sample_brick_valid_mask(g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_points"]),
                              g[f"{pre}_mask"])


def test_stokes_rk2_bit_exact(micro_golden):
    g = micro_golden
    out = O.stokes_rk2_brick(g["det_coeffs"], 0.05, g["det_initial"]).reshape(g["det_step"].shape)
    assert np.array_equal(out, g["det_step"])
    out = O.stokes_rk2_brick(g["det_coeffs"], 0.3, np.array([0.5, -0.1, 0.2, 0.05])).reshape(g["det_step"].shape)
    assert np.array_equal(out, g["det_step_broadcast"])
    assert np.array_equal(O.stokes_rk2_brick(g["rand_rk2_coeffs"], 0.11, g["rand_rk2_initial"]), g["rand_rk2_step"])


def test_reference_known_answers():
    """Known answers of the reference's own tests."""
    # native/core/src/lib.rs:406-414: scalar absorption -> I = 0.0975
    out = O.stokes_rk2_brick([1.0, 0, 0, 0, 0.5, 0, 0, 0, 0, 0, 0], 0.1, [0.0, 0, 0, 0])
    assert abs(out[0, 0] - 0.0975) < 1e-12 and np.all(out[0, 1:] == 0.0)
    # lib.rs:421-434: centre of the linear 2x2x2 fixture -> 55.5 / 55.51
    s = O.sample_brick_trilinear(rust_linear_fixture(), [0.0, 1.0], [0.0, 1.0], [0.0, 1.0], [0.5, 0.5, 0.5])
    assert abs(s[0, 0] - 55.5) < 1e-12 and abs(s[0, 10] - 55.51) < 1e-12
    # lib.rs:436-448: NaN outside the nonperiodic domain
    s = O.sample_brick_trilinear(rust_linear_fixture(), [0.0, 1.0], [0.0, 1.0], [0.0, 1.0],
                                 [-0.1, 0.5, 0.5, 0.5, 1.1, 0.5])
    assert np.all(np.isnan(s))
    # test_native_sampler_parity.py:57-65: 30.75 + k * 0.125
    c, rg, tg, pg = linear_coeff_fixture()
    s = O.sample_brick_trilinear(c, rg, tg, pg, [[0.25, 0.5, 0.75]])
    np.testing.assert_allclose(s[0], 30.75 + np.arange(11) * 0.125, rtol=1e-12, atol=1e-12)
    # :86-100 mask ignores phi
    m = O.sample_brick_valid_mask(rg, tg, [[0.5, 0.5, 0.5], [-0.1, 0.5, 0.5], [0.5, 1.1, 0.5], [0.5, 0.5, 100.0]])
    assert m.tolist() == [True, False, False, True]
    # :103-111 periodic wrap
    c4, rg, tg, pg = linear_coeff_fixture(4)
    a = O.sample_brick_trilinear(c4, rg, tg, pg, [[0.5, 0.5, math.pi / 4]])
    b = O.sample_brick_trilinear(c4, rg, tg, pg, [[0.5, 0.5, 2 * math.pi + math.pi / 4]])
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_kerr_geometry(kerr_golden):
    k = kerr_golden
    n = k["rhs_states"].shape[0]
    for i in range(n):
        r, th, a = k["rhs_states"][i, 1], k["rhs_states"][i, 2], k["rhs_a"][i]
        assert np.array_equal(O.metric_con(r, th, a), k["gcon_out"][i])
        assert np.array_equal(O.metric_cov(r, th, a), k["gcov_out"][i])
        rhs = O.geodesic_rhs(k["rhs_states"][i], a, k["rhs_pt"][i], k["rhs_pphi"][i])
        np.testing.assert_allclose(rhs, k["rhs_out"][i], rtol=1e-13, atol=1e-300)
        y = O.rk2_step(k["rhs_states"][i], k["rk2_h"][i], a, k["rhs_pt"][i], k["rhs_pphi"][i])
        np.testing.assert_allclose(y, k["rk2_out"][i], rtol=1e-13, atol=1e-300)
        h = O.hamiltonian(k["rhs_states"][i], a, k["rhs_pt"][i], k["rhs_pphi"][i])
        assert abs(h - k["ham_out"][i]) <= 1e-13 * max(1.0, abs(k["ham_out"][i]))


def test_camera_rays(kerr_golden):
    k = kerr_golden
    for i, (r, inc, fov, a, nx, ny, asp, roll) in enumerate(k["cam_params"]):
        v = O.make_view(spin_a=a, r_obs=r, theta_obs=math.radians(inc), phi_obs=0.0, fov_y_deg=fov, roll_deg=roll)
        y0, pt, pp = O.camera_ray(v, nx, ny, asp)
        assert np.array_equal(y0, k["cam_y0"][i]) and pt == k["cam_pt"][i] and pp == k["cam_pphi"][i]
        # test_kerr.py:34-37: camera rays are null
        assert abs(O.hamiltonian(y0, a, pt, pp)) < 1e-11


@pytest.mark.parametrize("name", ["c1", "c1_long", "near"])
def test_ray_loop_matches_reference_composition(ray_golden, name):
    g = ray_golden
    _, v = golden_view(g, name)
    img, steps, status, drift = O.render(v, g["brick_coeffs"], g["brick_r"], g["brick_theta"], g["brick_phi"],
                                         stop_at_tau=False, threads=2)
    ref = g[f"{name}_stokes"]
    np.testing.assert_allclose(img, ref, rtol=1e-11, atol=1e-12)
    assert np.array_equal(steps, g[f"{name}_steps"])
    assert np.array_equal(status, g[f"{name}_status"])
    d0 = g[f"{name}_h_drift"]
    np.testing.assert_allclose(drift, d0, rtol=1e-4, atol=1e-12)


def test_config1_is_all_zero(ray_golden):
    """The CPU-runnable configuration as stated (64 steps from r_obs = 1000 M)
    never reaches the brick: its image is exactly zero."""
    assert np.count_nonzero(ray_golden["c1_stokes"]) == 0
    assert np.all(ray_golden["c1_status"] == 0)


def test_stop_at_tau_does_not_change_stokes(ray_golden):
    g = ray_golden
    _, v = golden_view(g, "near")
    full = O.render(v, g["brick_coeffs"], g["brick_r"], g["brick_theta"], g["brick_phi"], stop_at_tau=False)[0]
    cut = O.render(v, g["brick_coeffs"], g["brick_r"], g["brick_theta"], g["brick_phi"], stop_at_tau=True)[0]
    assert np.array_equal(full, cut)
