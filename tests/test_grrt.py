"""The physical polarized GRRT renderer (polarized_renderer.render_stokes_image,
python/blackhole_sim/polarized_renderer.py:31-70): the oracle (oracle/grrt.py)
and the GPU kernel (bhn_grrt_render) against the reference's own image of a
seeded snapshot (tests/golden/grrt.npz), with RK2 and exact Stokes steps."""

from __future__ import annotations

from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import grrt as G
from oracle import oracle as O


@pytest.fixture(scope="module")
def golden():
    with np.load(Path(__file__).parent / "golden" / "grrt.npz") as z:
        return {k: z[k] for k in z}


def _fields(g):
    return np.concatenate([g["in_rho"][..., None], g["in_theta_e"][..., None], g["in_pressure"][..., None],
                           g["in_b_con"], g["in_u_con"]], axis=-1)


def _oracle_view(g, width=4, height=3):
    cam = g["cam"]
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = float(g["in_spin_a"]), cam[0], cam[1], cam[2]
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam[3], cam[4], width, height
    return v


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("exact,pix", [(False, (1, 2)), (True, (3, 0))])
def test_oracle_matches_reference(golden, exact, pix):
    px, py = pix
    scaling = dict(rho_cgs_per_code=float(golden["in_rho_cgs_per_code"]),
                   b_gauss_per_code=float(golden["in_b_gauss_per_code"]))
    S, (tau, emit, valid) = G.trace_pixel(_oracle_view(golden), _fields(golden), golden["in_r"], golden["in_theta"],
                                          golden["in_phi"], scaling, 230e9, 0.1, 900, 220.0,
                                          length_cm=float(golden["in_rg_cm"]), exact=exact, px=px, py=py)
    ref = golden["stokes_exact" if exact else "stokes_rk2"][py, px]
    assert emit > 0 and valid >= emit
    assert _rel(S, ref) <= 1e-12


def _snapshot(g):
    return SimpleNamespace(r=g["in_r"], theta=g["in_theta"], phi=g["in_phi"], rho=g["in_rho"], theta_e=g["in_theta_e"],
                           pressure=g["in_pressure"], b_con=g["in_b_con"], u_con=g["in_u_con"],
                           spin_a=float(g["in_spin_a"]))


def _scaling(g):
    return SimpleNamespace(rho_cgs_per_code=float(g["in_rho_cgs_per_code"]), b_gauss_per_code=float(g["in_b_gauss_per_code"]),
                           mean_molecular_weight_per_electron=1.0, rg_cm=float(g["in_rg_cm"]), flux_scale_jy=1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [False, True])
def test_gpu_matches_reference_image(golden, exact):
    from blackhole_native import grrt

    cam = golden["cam"]
    cfg = grrt.PolarizedRenderConfig(width=4, height=3, camera=grrt.LocalCamera(*cam), step=0.1, max_steps=900,
                                     transfer=grrt.PolarizedTransferConfig(use_exact_matrix_step=exact))
    img = grrt.render_stokes_image(cfg, _snapshot(golden), _scaling(golden))
    ref = golden["stokes_exact" if exact else "stokes_rk2"]
    assert img.shape == (3, 4, 4)
    for py in range(3):
        for px in range(4):
            assert _rel(img[py, px], ref[py, px]) <= 1e-10, (px, py)


@pytest.mark.gpu
def test_gpu_larger_image_against_oracle(golden):
    """A 24 x 16 image (warps over many rays): three pixels against the oracle,
    diagnostics consistent with the image."""
    from blackhole_native import grrt

    cam = golden["cam"]
    cfg = grrt.PolarizedRenderConfig(width=24, height=16, camera=grrt.LocalCamera(*cam), step=0.1, max_steps=900)
    img, diag = grrt.render_stokes_image_device(cfg, _snapshot(golden), _scaling(golden), diagnostics=True)
    img, diag = img.cpu().numpy(), diag.cpu().numpy()
    assert np.all(np.isfinite(img))
    emit, valid = diag[..., 1], diag[..., 2]
    assert np.all(valid >= emit) and np.all((img[..., 0] != 0) == (emit > 0))
    scaling = dict(rho_cgs_per_code=float(golden["in_rho_cgs_per_code"]),
                   b_gauss_per_code=float(golden["in_b_gauss_per_code"]))
    for px, py in ((0, 0), (11, 7), (23, 15)):
        S, (tau, e, va) = G.trace_pixel(_oracle_view(golden, 24, 16), _fields(golden), golden["in_r"], golden["in_theta"],
                                        golden["in_phi"], scaling, 230e9, 0.1, 900, 220.0,
                                        length_cm=float(golden["in_rg_cm"]), px=px, py=py)
        assert e == diag[py, px, 1] and va == diag[py, px, 2]
        assert _rel(img[py, px], S) <= 1e-10 if np.any(S) else not np.any(img[py, px])
        assert abs(tau - diag[py, px, 0]) <= 1e-10 * max(tau, 1e-300)


def test_seeded_snapshot_is_deterministic():
    from blackhole_native import grrt

    a, b = grrt.seeded_snapshot(6, 4, 5, seed=3), grrt.seeded_snapshot(6, 4, 5, seed=3)
    assert a.rho.shape == (6, 4, 5) and a.b_con.shape == (6, 4, 5, 4) and a.u_con.shape == (6, 4, 5, 4)
    assert np.array_equal(a.rho, b.rho) and np.array_equal(a.b_con, b.b_con)
    assert np.all(a.rho > 0) and np.all((a.theta_e >= 1.0) & (a.theta_e <= 60.0))
    assert np.all(np.diff(a.r) > 0) and a.theta[0] > 0 and a.theta[-1] < np.pi and a.phi[-1] < 2 * np.pi
    f = grrt.snapshot_fields(a)
    assert f.shape == (6, 4, 5, 11) and np.array_equal(f[..., 3:7], a.b_con)
    with pytest.raises(ValueError):
        grrt.seeded_snapshot(1, 4, 5)


@pytest.mark.gpu
def test_gpu_seeded_snapshot_device_reuse_against_oracle():
    """A seeded snapshot kept on the device (DeviceSnapshot) renders the same
    image into a caller's buffer as the host-snapshot call, and its pixels
    match the oracle."""
    import torch

    from blackhole_native import grrt

    snap = grrt.seeded_snapshot(16, 8, 12, seed=4)
    scaling = grrt.PhysicalScaling(mass_bh_g=8.54e39, distance_cm=2.57e22, rho_cgs_per_code=3.0e-18,
                                   b_gauss_per_code=25.0)
    cam = grrt.LocalCamera.from_degrees(r=30.0, inclination_degrees=70.0, fov_y_degrees=30.0)
    cfg = grrt.PolarizedRenderConfig(width=12, height=8, camera=cam, step=0.1, max_steps=900)
    host = grrt.render_stokes_image(cfg, snap, scaling)
    ds = grrt.DeviceSnapshot(snap)
    out = torch.full((8, 12, 4), float("nan"), dtype=torch.float64, device="cuda")
    got = grrt.render_stokes_image_device(cfg, ds, scaling, out=out)
    assert got is out and np.array_equal(out.cpu().numpy(), host)
    with pytest.raises(ValueError, match="out must be"):
        grrt.render_stokes_image_device(cfg, ds, scaling, out=out[:4])
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = snap.spin_a, cam.r, cam.theta, cam.phi
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam.fov_y_degrees, cam.roll_degrees, 12, 8
    sc = dict(rho_cgs_per_code=scaling.rho_cgs_per_code, b_gauss_per_code=scaling.b_gauss_per_code)
    for px, py in ((5, 3), (11, 0)):
        S, _ = G.trace_pixel(v, grrt.snapshot_fields(snap), snap.r, snap.theta, snap.phi, sc, 230e9, 0.1, 900, 220.0,
                             length_cm=scaling.rg_cm, exact=False, px=px, py=py)
        assert _rel(host[py, px], S) <= 1e-10 if np.any(S) else not np.any(host[py, px])


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [False, True])
def test_gpu_chunk_does_not_change_the_image(golden, exact):
    """The renderer lists `chunk` emitting segments per ray and round; one
    segment per round, three, and the default give the same image and
    diagnostics bit for bit (a tiny optical-depth cutoff makes rays end
    mid-round, after segments their trace already listed)."""
    from blackhole_native import grrt

    cam = golden["cam"]
    snap, sc = _snapshot(golden), _scaling(golden)
    for max_tau in (30.0, 1e-6):
        tr = grrt.PolarizedTransferConfig(use_exact_matrix_step=exact, max_optical_depth=max_tau)
        cfg = grrt.PolarizedRenderConfig(width=12, height=8, camera=grrt.LocalCamera(*cam), step=0.1, max_steps=900,
                                         transfer=tr)
        ref, ref_d = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg, snap, sc, diagnostics=True))
        if max_tau < 1.0:
            assert np.any(ref_d[..., 7] == 4)  # some rays end opaque
        for chunk in (1, 3):
            img, d = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg, snap, sc, diagnostics=True,
                                                                             chunk=chunk))
            assert np.array_equal(img, ref) and np.array_equal(d, ref_d), (max_tau, chunk)


@pytest.mark.gpu
def test_gpu_edge_cases(golden):
    """No steps at all; a camera inside the snapshot whose rays run out of
    steps while they emit (against the oracle); the renderer's argument checks."""
    from blackhole_native import grrt

    snap, sc = _snapshot(golden), _scaling(golden)
    cam = golden["cam"]
    cfg0 = grrt.PolarizedRenderConfig(width=5, height=4, camera=grrt.LocalCamera(*cam), step=0.1, max_steps=0)
    img, d = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg0, snap, sc, diagnostics=True))
    assert not np.any(img) and np.all(d[..., 6] == 0) and np.all(d[..., 7] == 0)  # 0 steps, BHN_RAY_MAX_STEPS

    inside = grrt.LocalCamera.from_degrees(r=12.0, inclination_degrees=80.0, fov_y_degrees=50.0)
    cfg = grrt.PolarizedRenderConfig(width=6, height=4, camera=inside, step=0.1, max_steps=37)
    img, d = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg, snap, sc, diagnostics=True, chunk=5))
    assert np.all(d[..., 6] <= 37) and np.any(d[..., 7] == 0) and np.any(d[..., 1] > 0)
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = float(golden["in_spin_a"]), inside.r, inside.theta, inside.phi
    v.fov_y_deg, v.roll_deg, v.width, v.height = inside.fov_y_degrees, 0.0, 6, 4
    scaling = dict(rho_cgs_per_code=float(golden["in_rho_cgs_per_code"]),
                   b_gauss_per_code=float(golden["in_b_gauss_per_code"]))
    for px, py in ((0, 0), (3, 2), (5, 3)):
        S, (tau, e, va) = G.trace_pixel(v, _fields(golden), golden["in_r"], golden["in_theta"], golden["in_phi"],
                                        scaling, 230e9, 0.1, 37, 220.0, length_cm=float(golden["in_rg_cm"]),
                                        px=px, py=py)
        assert e == d[py, px, 1] and va == d[py, px, 2]
        assert _rel(img[py, px], S) <= 1e-10 if np.any(S) else not np.any(img[py, px])

    with pytest.raises(ValueError, match="step must be finite and positive"):
        grrt.render_stokes_image_device(grrt.PolarizedRenderConfig(width=2, height=2, step=0.0), snap, sc)
    with pytest.raises(ValueError, match="chunk must be positive"):
        grrt.render_stokes_image_device(cfg, snap, sc, chunk=0)


def test_stokes_to_rgb_and_npz_match_the_reference(tmp_path):
    """polarized_renderer.stokes_to_rgb / save_stokes_npz against the
    reference's own outputs (tests/golden/stokes_rgb.npz)."""
    from blackhole_native import grrt

    with np.load(Path(__file__).parent / "golden" / "stokes_rgb.npz") as z:
        g = {k: z[k] for k in z}
    assert np.array_equal(grrt.stokes_to_rgb(g["rgb_in"]), g["rgb_out"])
    assert np.array_equal(grrt.stokes_to_rgb(g["rgb_in"], gamma=1.8), g["rgb_out_g18"])
    assert np.array_equal(grrt.stokes_to_rgb(g["rgb_dark_in"]), g["rgb_dark_out"])
    out = tmp_path / "a" / "b" / "img.npz"
    grrt.save_stokes_npz(g["rgb_in"].astype(np.float32), out)
    with np.load(out) as z:
        assert list(z.keys()) == ["stokes"] and z["stokes"].dtype == np.float64
        assert np.array_equal(z["stokes"], g["rgb_in"].astype(np.float32).astype(np.float64))


@pytest.mark.gpu
def test_gpu_outbound_exit_keeps_the_image(golden):
    """A ray past the snapshot's outer radius moving out for good ends there
    (status 5): the image and the optical-depth, segment and redshift columns
    equal a full trace's bit for bit, on the golden scene (with and without a
    cutoff that ends rays) and on a seeded 32 x 16 x 32 snapshot seen from
    r = 55 M; outbound rays are ones the full trace ends as escaped or at
    max_steps, after no more steps."""
    from blackhole_native import grrt

    sc = _scaling(golden)
    seeded = grrt.seeded_snapshot(32, 16, 32, 0.9375, 3)
    scenes = []
    for max_tau in (30.0, 1e-6):
        tr = grrt.PolarizedTransferConfig(max_optical_depth=max_tau)
        scenes.append((grrt.PolarizedRenderConfig(width=12, height=8, camera=grrt.LocalCamera(*golden["cam"]),
                                                  step=0.1, max_steps=900, transfer=tr), _snapshot(golden)))
    scenes.append((grrt.PolarizedRenderConfig(width=24, height=14), seeded))
    outbound = 0
    for cfg, snap in scenes:
        img, d = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg, snap, sc, diagnostics=True))
        ref, rd = (t.cpu().numpy() for t in grrt.render_stokes_image_device(cfg, snap, sc, diagnostics=True,
                                                                           full_trace=True))
        assert np.array_equal(img, ref) and np.array_equal(d[..., :6], rd[..., :6])
        out = d[..., 7] == 5
        assert np.array_equal(d[..., 7][~out], rd[..., 7][~out]) and np.all(np.isin(rd[..., 7][out], (0, 2)))
        assert np.all(d[..., 6] <= rd[..., 6]) and not np.any(rd[..., 7] == 5)
        outbound += int(out.sum())
    assert outbound > 0
