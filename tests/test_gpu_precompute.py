"""GPU coefficient-brick precompute (bhn_brick_precompute) against the
reference's own precompute_coefficient_bricks outputs (tests/golden/
brick_precompute.npz) and the oracle (oracle/synchrotron.py).

FP64 throughout: float64 bricks agree with the reference to 1e-12 of each
channel's largest value; float32 bricks to float32 rounding."""

from __future__ import annotations

from dataclasses import replace
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest
import torch

import blackhole_native as bn
from blackhole_native import synchrotron as syn
from oracle import synchrotron as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    with np.load(Path(__file__).parent / "golden" / "brick_precompute.npz") as z:
        g = {k: z[k] for k in z}
    snap = SimpleNamespace(r=g["in_r"], theta=g["in_theta"], phi=g["in_phi"], rho=g["in_rho"],
                           theta_e=g["in_theta_e"], b_con=g["in_b_con"], spin_a=float(g["in_spin_a"]))
    scaling = SimpleNamespace(rho_cgs_per_code=float(g["in_rho_cgs_per_code"]),
                              b_gauss_per_code=float(g["in_b_gauss_per_code"]),
                              mean_molecular_weight_per_electron=float(g["in_mu_e"]))
    return g, snap, scaling


def _err(out, ref):
    scale = np.maximum(np.abs(ref).max(axis=tuple(range(ref.ndim - 1))), 1e-300)
    return float(np.max(np.abs(out - ref) / scale))


@pytest.mark.parametrize("nu,tag", [(230e9, "230"), (86e9, "86")])
def test_precompute_matches_reference(golden, nu, tag):
    g, snap, scaling = golden
    b64 = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=nu, dtype="float64")
    ref = g[f"coeffs64_{tag}"]
    assert b64.coeffs.dtype == np.float64 and b64.coeffs.shape == ref.shape
    assert np.array_equal(b64.r, g["in_r"]) and np.array_equal(b64.phi, g["in_phi"])
    assert np.array_equal(b64.coeffs == 0.0, ref == 0.0)
    assert _err(b64.coeffs, ref) <= 1e-12
    nz = ref != 0.0
    assert np.max(np.abs(b64.coeffs[nz] - ref[nz]) / np.abs(ref[nz])) <= 1e-11
    b32 = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=nu)
    assert b32.coeffs.dtype == np.float32
    np.testing.assert_allclose(b32.coeffs, g[f"coeffs32_{tag}"], rtol=2e-7, atol=0)


def test_precompute_stride(golden):
    g, snap, scaling = golden
    b = bn.precompute_coefficient_bricks(snap, scaling, dtype="float64", stride=2)
    assert b.coeffs.shape == g["coeffs64_230_stride2"].shape
    assert _err(b.coeffs, g["coeffs64_230_stride2"]) <= 1e-12
    with pytest.raises(ValueError, match="stride"):
        bn.precompute_coefficient_bricks(snap, scaling, stride=0)


def test_single_components_and_model_parameters(golden):
    """Each component alone, and non-default parameters, against the oracle."""
    g, snap, scaling = golden
    th = syn.ThermalSynchrotronCoefficients(gamma_grid_size=97, pitch_nodes=7, faraday_conversion_scale=0.5)
    nt = syn.NonthermalPowerLawSynchrotronCoefficients(p=2.8, gamma_min=4.0, gamma_max=3e4, nonthermal_fraction=0.1,
                                                       gamma_grid_size=61, pitch_nodes=5, faraday_scale=0.3)
    args = (g["in_rho"], g["in_theta_e"], g["in_b_con"])
    cells = np.ndindex(g["in_rho"].shape)
    want_th = np.zeros(g["in_rho"].shape + (11,))
    want_nt = np.zeros_like(want_th)
    for idx in cells:
        n_e, te, b, chi = S.cell_frame(float(args[0][idx]), float(args[1][idx]), args[2][idx],
                                       scaling.rho_cgs_per_code, scaling.b_gauss_per_code)
        want_th[idx] = S.thermal(n_e, te, b, chi, 150e9, dict(vars(th)))
        want_nt[idx] = S.nonthermal(n_e, te, b, chi, 150e9, dict(vars(nt)))
    got_th = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=150e9, dtype="float64", coeff_model=th).coeffs
    got_nt = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=150e9, dtype="float64", coeff_model=nt).coeffs
    assert _err(got_th, want_th) <= 1e-12
    assert _err(got_nt, want_nt) <= 1e-12
    both = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=150e9, dtype="float64",
                                            coeff_model=syn.HybridSynchrotronCoefficients(th, nt)).coeffs
    assert _err(both, want_th + want_nt) <= 1e-12


def test_device_brick_feeds_the_renderer():
    """A 64 x 32 x 48 snapshot precomputed straight into the renderer's records
    renders the same image as the host brick (same float32 values)."""
    rng = np.random.default_rng(3)
    a = 0.9375
    r = np.geomspace(1.05 * bn.horizon_radius(a), 40.0, 64)
    theta = (np.arange(32) + 0.5) * np.pi / 32
    phi = np.linspace(0.0, 2 * np.pi, 48, endpoint=False)
    shape = (64, 32, 48)
    rho = np.exp(-((r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(theta)[None, :, None] ** 2) * np.ones(shape)
    snap = SimpleNamespace(r=r, theta=theta, phi=phi, rho=rho, theta_e=np.full(shape, 20.0),
                           b_con=rng.normal(0.0, 1.0, shape + (4,)), spin_a=a)
    scaling = SimpleNamespace(rho_cgs_per_code=3e-18, b_gauss_per_code=25.0, mean_molecular_weight_per_electron=1.0)
    host = bn.precompute_coefficient_bricks(snap, scaling)
    assert np.all(np.isfinite(host.coeffs)) and np.all(host.coeffs[..., 0] >= 0) and host.coeffs[..., 0].max() > 0
    db = bn.precompute_device_brick(snap, scaling)
    view = bn.View(64, 48, max_steps=3000)
    a_img = bn.render(db, view).image()
    b_img = bn.render(bn.DeviceBrick(host), view).image()
    assert torch.equal(a_img, b_img)


def test_rejects_bad_models(golden):
    g, snap, scaling = golden
    with pytest.raises(ValueError, match="gamma grids"):
        bn.precompute_coefficient_bricks(snap, scaling, coeff_model=syn.ThermalSynchrotronCoefficients(pitch_nodes=0))
    with pytest.raises(ValueError, match="gamma_min"):
        bn.precompute_coefficient_bricks(
            snap, scaling, coeff_model=syn.NonthermalPowerLawSynchrotronCoefficients(gamma_min=10.0, gamma_max=5.0))
    with pytest.raises(ValueError, match="dtype"):
        bn.precompute_coefficient_bricks(snap, scaling, dtype="bfloat16")


def test_extreme_plasma_regimes_against_oracle():
    """Cells far from the fixtures' plasma: Theta_e from 1e-3 (nearly every
    thermal Lorentz-factor node in the kernel table's far tail, where the GPU
    skips it) to 1e3, |B| from 1e-3 to 1e3 code units, zero density; the
    float64 brick against the oracle cell by cell."""
    import itertools

    rng = np.random.default_rng(9)
    cells = []
    for te, bs, rho in itertools.product((1e-3, 0.05, 1.0, 30.0, 1e3), (1e-3, 1.0, 1e3), (0.0, 1e-3, 1.0)):
        for _ in range(2):
            b = rng.normal(size=4)
            b[1:] *= bs / np.linalg.norm(b[1:])
            cells.append((rho, te, b))
    cells += cells[: -len(cells) % 4]  # a [n][2][2] brick (grids need two values per axis)
    n = len(cells) // 4
    rho = np.array([c[0] for c in cells]).reshape(n, 2, 2)
    te = np.array([c[1] for c in cells]).reshape(n, 2, 2)
    bc = np.array([c[2] for c in cells]).reshape(n, 2, 2, 4)
    snap = SimpleNamespace(r=np.arange(n, dtype=np.float64) + 2.0, theta=np.array([1.0, 2.0]), phi=np.array([0.0, 3.0]),
                           rho=rho, theta_e=te, b_con=bc, spin_a=0.9)
    scaling = SimpleNamespace(rho_cgs_per_code=3e-18, b_gauss_per_code=25.0, mean_molecular_weight_per_electron=1.0)
    got = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=230e9, dtype="float64").coeffs
    ref = S.precompute(rho, te, bc, 230e9, 3e-18, 25.0, dtype="float64")
    assert np.array_equal(got == 0.0, ref == 0.0) and np.any(ref != 0.0)
    assert _err(got, ref) <= 1e-12
    nz = ref != 0.0
    assert np.max(np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])) <= 1e-10


def test_pipelined_host_path_equals_device_path():
    """A snapshot above the pipelining threshold: the host-to-host call (r
    slabs through pinned buffers on copy streams) returns exactly the
    device-resident result, for both output precisions."""
    from blackhole_native import grrt

    snap = grrt.seeded_snapshot(20, 256, 256, seed=3)   # 1.3M cells, 20 r shells
    scaling = SimpleNamespace(rho_cgs_per_code=3e-18, b_gauss_per_code=25.0, mean_molecular_weight_per_electron=1.0)
    assert snap.rho.size >= syn.PIPELINE_MIN_CELLS
    for dtype in ("float32", "float64"):
        host = bn.precompute_coefficient_bricks(snap, scaling, dtype=dtype)
        dev_out = syn.precompute_device_coefficients(snap, scaling, dtype=dtype)[3].cpu().numpy()
        assert host.coeffs.dtype == dev_out.dtype and np.array_equal(host.coeffs, dev_out)


def test_precompute_float16_and_stride(golden):
    """dtype="float16" (test_coefficient_bricks.py:30-35, coefficient_bricks.py:
    140-151): the float64 coefficients rounded once to float16, then
    nan_to_num(nan=0, posinf=finfo(float16).max, neginf=0); a float16 brick
    widens exactly to the renderer's float32 records."""
    g, snap, scaling = golden
    b = bn.precompute_coefficient_bricks(snap, scaling, nu_hz=230e9, dtype="float16", stride=2)
    ref64 = g["coeffs64_230_stride2"]
    with np.errstate(over="ignore"):
        want = np.nan_to_num(ref64.astype(np.float16), nan=0.0, posinf=np.finfo(np.float16).max, neginf=0.0)
    assert b.coeffs.dtype == np.float16 and b.coeffs.shape == want.shape and b.nu_hz == 230e9
    assert np.array_equal(b.coeffs, want)
    scaled = bn.BrickGrid(b.r, b.theta, b.phi, (ref64 * (1.0 / max(np.abs(ref64).max(), 1e-300))).astype(np.float16),
                          spin_a=b.spin_a)
    view = bn.View(24, 24, spin_a=b.spin_a, r_obs=30.0, inclination_deg=70.0, fov_y_deg=30.0, max_steps=900)
    img16 = bn.render(bn.DeviceBrick(scaled), view).image().cpu().numpy()
    wide = bn.BrickGrid(b.r, b.theta, b.phi, scaled.coeffs.astype(np.float32), spin_a=b.spin_a)
    img32 = bn.render(bn.DeviceBrick(wide), view).image().cpu().numpy()
    assert np.array_equal(img16, img32)
    with pytest.raises(ValueError, match="dtype"):
        bn.precompute_coefficient_bricks(snap, scaling, dtype="int8")
