"""CPU checks of the brick-precompute oracle (oracle/synchrotron.py) against
fixtures made by the reference's own precompute_coefficient_bricks
(python/blackhole_sim/coefficient_bricks.py:119-152, Hybrid model)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import synchrotron as S


@pytest.fixture(scope="module")
def golden():
    from pathlib import Path

    with np.load(Path(__file__).parent / "golden" / "brick_precompute.npz") as z:
        return {k: z[k] for k in z}


def _err(out, ref):
    """Largest error relative to each channel's largest magnitude."""
    scale = np.maximum(np.abs(ref).max(axis=tuple(range(ref.ndim - 1))), 1e-300)
    return float(np.max(np.abs(out - ref) / scale))


def test_kernel_table(golden):
    xs, F, G = S.kernel_table()
    assert np.array_equal(xs, golden["table_xs"])
    assert np.array_equal(F, golden["table_F"])
    big = golden["table_G"] > 1e-290
    np.testing.assert_allclose(G[big], golden["table_G"][big], rtol=1e-12)
    assert np.all(G[~big] < 1e-280)


@pytest.mark.parametrize("nu,tag", [(230e9, "230"), (86e9, "86")])
def test_precompute_matches_reference(golden, nu, tag):
    args = (golden["in_rho"], golden["in_theta_e"], golden["in_b_con"], nu, float(golden["in_rho_cgs_per_code"]),
            float(golden["in_b_gauss_per_code"]), float(golden["in_mu_e"]))
    out64 = S.precompute(*args, dtype="float64")
    ref = golden[f"coeffs64_{tag}"]
    assert np.array_equal(out64 == 0.0, ref == 0.0)          # exact zeros: zero field, j_V, alpha_V, rho_V
    assert _err(out64, ref) <= 1e-12
    nz = ref != 0.0
    assert np.max(np.abs(out64[nz] - ref[nz]) / np.abs(ref[nz])) <= 1e-11
    out32 = S.precompute(*args, dtype="float32")
    np.testing.assert_allclose(out32, golden[f"coeffs32_{tag}"], rtol=2e-7, atol=0)


def test_precompute_stride(golden):
    out = S.precompute(golden["in_rho"], golden["in_theta_e"], golden["in_b_con"], 230e9,
                       float(golden["in_rho_cgs_per_code"]), float(golden["in_b_gauss_per_code"]),
                       float(golden["in_mu_e"]), dtype="float64", stride=2)
    assert _err(out, golden["coeffs64_230_stride2"]) <= 1e-12


def test_kv_against_closed_form():
    """K_{1/2}(x) = sqrt(pi / (2x)) exp(-x) (DLMF 10.39.2) checks the quadrature."""
    x = np.array([1e-6, 1e-3, 0.1, 1.0, 7.0, 40.0, 300.0])
    np.testing.assert_allclose(S.kv(0.5, x), np.sqrt(np.pi / (2 * x)) * np.exp(-x), rtol=1e-12)
