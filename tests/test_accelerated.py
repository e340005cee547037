"""The reference's own brick renderer (accelerated_renderer.render_stokes_image_bricks
/ render_tile_stokes_bricks, python/blackhole_sim/accelerated_renderer.py:100-158:
fixed-step RK4, trilinear brick samples, RK2 or exact Stokes steps): the oracle
(oracle/bricktrace.py) and the GPU (bhn_brick_trace_render) against the
reference's own 5 x 4 images of a seeded brick (tests/golden/accel.npz).

The reference interpolates with float32 weights (its float32 grids under
NumPy's promotion rules) while oracle and GPU do it in float64: pixels agree
to 1e-6 relative (measured 3e-8)."""

from __future__ import annotations

from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import bricktrace as B
from oracle import oracle as O

TOL = 1e-6


@pytest.fixture(scope="module")
def golden():
    with np.load(Path(__file__).parent / "golden" / "accel.npz") as z:
        return {k: z[k] for k in z}


def _grids(g):
    return [g[k].astype(np.float32).astype(np.float64) for k in ("acc_r", "acc_theta", "acc_phi")]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _cases():
    for dt in ("float64", "float32"):
        for step in ("rk2", "exact"):
            for cut in ("full", "cut"):
                yield dt, step, cut


@pytest.mark.parametrize("dt,step,cut", [c for c in _cases() if c[2] == "cut" or c[1] == "rk2"])
def test_oracle_matches_reference(golden, dt, step, cut):
    rg, tg, pg = _grids(golden)
    cam = golden["acc_cam"]
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = 0.9375, cam[0], cam[1], cam[2]
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam[3], 0.0, 5, 4
    coeffs = golden["acc_coeffs"].astype(dt).astype(np.float64)
    ref = golden[f"acc_{dt}_{step}_{cut}"]
    for px, py in ((0, 0), (2, 1), (4, 3)):
        S, (tau, n) = B.trace_pixel_bricks(v, coeffs, rg, tg, pg, 0.1, 900, 220.0, length_cm=2.0, exact=step == "exact",
                                           max_tau=30.0 if cut == "full" else 0.006, px=px, py=py)
        assert n > 0 and _rel(S, ref[py, px]) <= TOL


def _config(acc, cam, step, cut):
    from blackhole_native import grrt

    tr = grrt.PolarizedTransferConfig(use_exact_matrix_step=step == "exact", affine_to_length_cm=2.0,
                                      max_optical_depth=30.0 if cut == "full" else 0.006)
    return acc.AcceleratedRenderConfig(width=5, height=4, camera=grrt.LocalCamera(cam[0], cam[1], cam[2], cam[3]),
                                       step=0.1, max_steps=900, transfer=tr)


@pytest.mark.gpu
@pytest.mark.parametrize("dt,step,cut", list(_cases()))
def test_gpu_matches_reference_image(golden, dt, step, cut):
    from blackhole_native import accelerated as acc

    bricks = SimpleNamespace(r=golden["acc_r"], theta=golden["acc_theta"], phi=golden["acc_phi"],
                             coeffs=golden["acc_coeffs"].astype(dt))
    snap = SimpleNamespace(spin_a=0.9375)
    img, diag = acc.render_stokes_image_bricks_device(_config(acc, golden["acc_cam"], step, cut), snap, bricks,
                                                      diagnostics=True)
    img, diag = img.cpu().numpy(), diag.cpu().numpy()
    ref = golden[f"acc_{dt}_{step}_{cut}"]
    assert img.shape == (4, 5, 4) and np.all(np.isfinite(img))
    for py in range(4):
        for px in range(5):
            assert _rel(img[py, px], ref[py, px]) <= TOL, (px, py)
    if cut == "cut":
        assert np.any(diag[..., 3] == 4) and np.all(diag[..., 0][diag[..., 3] == 4] >= 0.006)


@pytest.mark.gpu
def test_gpu_tile_and_oracle(golden):
    """render_tile_stokes_bricks against the reference's tile, and a larger
    image's pixels (with sampled-segment counts) against the oracle."""
    from blackhole_native import accelerated as acc
    from blackhole_native.tiles import RenderTile

    cam = golden["acc_cam"]
    bricks = SimpleNamespace(r=golden["acc_r"], theta=golden["acc_theta"], phi=golden["acc_phi"],
                             coeffs=golden["acc_coeffs"].astype(np.float32))
    snap = SimpleNamespace(spin_a=0.9375)
    cfg = _config(acc, cam, "rk2", "full")
    cfg = acc.AcceleratedRenderConfig(width=5, height=4, camera=cfg.camera, step=0.1, max_steps=900)
    block = acc.render_tile_stokes_bricks(cfg, snap, bricks, RenderTile(level=0, y0=1, x0=2, x1=5, y1=3))
    assert block.shape == (2, 3, 4) and _rel(block, golden["acc_float32_tile"]) <= TOL

    big = acc.AcceleratedRenderConfig(width=24, height=16, camera=cfg.camera, step=0.1, max_steps=900,
                                      transfer=_config(acc, cam, "rk2", "full").transfer)
    img, diag = (t.cpu().numpy() for t in acc.render_stokes_image_bricks_device(big, snap, bricks, diagnostics=True))
    rg, tg, pg = _grids(golden)
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = 0.9375, cam[0], cam[1], cam[2]
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam[3], 0.0, 24, 16
    coeffs = golden["acc_coeffs"].astype(np.float32).astype(np.float64)
    for px, py in ((0, 0), (11, 7), (23, 15)):
        S, (tau, n) = B.trace_pixel_bricks(v, coeffs, rg, tg, pg, 0.1, 900, 220.0, length_cm=2.0, px=px, py=py)
        assert n == diag[py, px, 1]
        assert _rel(img[py, px], S) <= 1e-10 if np.any(S) else not np.any(img[py, px])


def _golden_bricks(golden, dt=np.float32):
    return SimpleNamespace(r=golden["acc_r"], theta=golden["acc_theta"], phi=golden["acc_phi"],
                           coeffs=golden["acc_coeffs"].astype(dt))


def test_host_validation_before_any_device_work(golden):
    """Bad bricks, configs and tiles raise ValueError, GPU or not: all on the
    host before any device work, except a non-finite coefficient, which a GPU
    finds in the uploaded brick (the same error; test_gpu_edge_cases)."""
    from dataclasses import replace

    from blackhole_native import accelerated as acc
    from blackhole_native.tiles import RenderTile

    snap = SimpleNamespace(spin_a=0.9375)
    cfg = _config(acc, golden["acc_cam"], "rk2", "full")
    good = _golden_bricks(golden)
    bad_shape = SimpleNamespace(**{**vars(good), "coeffs": good.coeffs[:, :, :-1]})
    with pytest.raises(ValueError, match="coeffs must have shape"):
        acc.render_stokes_image_bricks(cfg, snap, bad_shape)
    nonfinite = SimpleNamespace(**{**vars(good), "coeffs": good.coeffs.copy()})
    nonfinite.coeffs[1, 1, 1, 4] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        acc.render_stokes_image_bricks(cfg, snap, nonfinite)
    unsorted = SimpleNamespace(**{**vars(good), "r": good.r[::-1].copy()})
    with pytest.raises(ValueError, match="strictly increasing"):
        acc.render_stokes_image_bricks(cfg, snap, unsorted)
    with pytest.raises(ValueError, match="step must be"):
        acc.render_stokes_image_bricks(replace(cfg, step=0.0), snap, good)
    with pytest.raises(ValueError, match="max_steps"):
        acc.render_stokes_image_bricks(replace(cfg, max_steps=-1), snap, good)
    with pytest.raises(ValueError, match="outside"):
        acc.render_tile_stokes_bricks(cfg, snap, good, RenderTile(level=0, y0=0, x0=3, x1=6, y1=2))


def test_c_abi_rejects_bad_arguments_before_device_work():
    """bhn_brick_trace_render checks pointers, grid sizes and the config on
    the host and returns BHN_ERR_VALUE with a message, launching nothing."""
    import ctypes

    from blackhole_native import _lib
    from blackhole_native import accelerated as acc

    L = acc._declare()
    buf = (ctypes.c_double * 64)()
    p = ctypes.addressof(buf)
    v = _lib.ViewStruct()
    c = acc.BrickTraceConfigStruct(step=0.1, escape_radius=220.0, length_cm=1.0, max_optical_depth=30.0, max_steps=10,
                                   exact_step=0)

    def call(nr=4, cfg=c, out=p):
        return L.bhn_brick_trace_render(p, p, nr, p, 4, p, 4, ctypes.byref(v), ctypes.byref(cfg), p, 512, out, None,
                                        None)

    assert call(out=None) == 1 and b"missing" in L.bhn_last_error()
    assert call(nr=1) == 1 and b"at least 2" in L.bhn_last_error()
    for field, value, msg in (("step", 0.0, b"step"), ("step", float("nan"), b"step"), ("max_steps", -1, b"max_steps"),
                              ("length_cm", float("inf"), b"finite"), ("coeff_layout", 3, b"layout")):
        bad = acc.BrickTraceConfigStruct.from_buffer_copy(c)
        setattr(bad, field, value)
        assert call(cfg=bad) == 1 and msg in L.bhn_last_error(), field
    rec = acc.BrickTraceConfigStruct.from_buffer_copy(c)
    rec.coeff_layout = acc.BRICK_F32X12
    assert L.bhn_brick_trace_render(p + 8 if p % 16 == 0 else p, p, 4, p, 4, p, 4, ctypes.byref(v), ctypes.byref(rec),
                                    p, 512, p, None, None) == 1 and b"16-byte" in L.bhn_last_error()


def test_config_struct_layout_matches_ctypes(tmp_path):
    import ctypes
    import shutil
    import subprocess

    from blackhole_native import accelerated as acc

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    include = Path(__file__).resolve().parents[1] / "include"
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "blackhole_native.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(bhn_brick_trace_config),'
                   ' offsetof(bhn_brick_trace_config, max_steps), offsetof(bhn_brick_trace_config, exact_step),'
                   ' offsetof(bhn_brick_trace_config, full_trace), offsetof(bhn_brick_trace_config, coeff_layout));'
                   ' return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(include), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    S = acc.BrickTraceConfigStruct
    assert got == [ctypes.sizeof(S), S.max_steps.offset, S.exact_step.offset, S.full_trace.offset,
                   S.coeff_layout.offset]


@pytest.mark.gpu
def test_gpu_edge_cases(golden):
    """max_steps = 0 traces nothing (a zero image, status max_steps); an empty
    tile gives an empty block, as the reference's loop over no pixels."""
    from dataclasses import replace

    from blackhole_native import accelerated as acc
    from blackhole_native.tiles import RenderTile

    snap = SimpleNamespace(spin_a=0.9375)
    cfg = _config(acc, golden["acc_cam"], "rk2", "full")
    nonfinite = _golden_bricks(golden)
    nonfinite.coeffs = nonfinite.coeffs.copy()
    nonfinite.coeffs[1, 1, 1, 4] = np.inf
    with pytest.raises(ValueError, match="non-finite"):
        acc.render_stokes_image_bricks(cfg, snap, nonfinite)
    img, diag = (t.cpu().numpy() for t in acc.render_stokes_image_bricks_device(
        replace(cfg, max_steps=0), snap, _golden_bricks(golden), diagnostics=True))
    assert not np.any(img) and not np.any(diag[..., :3]) and np.all(diag[..., 3] == 0)  # BHN_RAY_MAX_STEPS
    block = acc.render_tile_stokes_bricks(cfg, snap, _golden_bricks(golden), RenderTile(level=0, y0=2, x0=1, x1=4, y1=2))
    assert block.shape == (0, 3, 4)


# ---- the reference's own regression test (test_accelerated_renderer.py:17-78) as data
@pytest.fixture(scope="module")
def regression():
    with np.load(Path(__file__).parent / "golden" / "accel_regression.npz") as z:
        return {k: z[k] for k in z}


def _reg_inputs(g):
    from blackhole_native import grrt

    snap = grrt.Snapshot(**{k: g[f"snap_{k}"] for k in ("r", "theta", "phi", "rho", "theta_e", "pressure", "b_con",
                                                           "u_con")}, spin_a=float(g["snap_spin_a"]))
    scaling = grrt.PhysicalScaling(**{k: float(g[f"scaling_{k}"]) for k in (
        "mass_bh_g", "distance_cm", "rho_cgs_per_code", "b_gauss_per_code", "ion_to_electron_temperature_ratio",
        "mean_molecular_weight_per_electron", "flux_scale_jy")})
    return snap, scaling


def test_regression_metrics_match_the_reference(regression):
    """compare_reference_vs_bricks on the reference's own two images gives its metrics."""
    from blackhole_native import accelerated as acc

    reg = acc.compare_reference_vs_bricks(regression["reg_ref"], regression["reg_cand"])
    m = reg.metrics
    assert np.array_equal(np.array([m.max_abs, m.mean_abs, m.rmse, m.psnr_db]), regression["reg_metrics"])
    assert reg.candidate.shape == reg.reference.shape == (2, 3, 4) and len(m.sha256) == 64
    with pytest.raises(ValueError, match="shape mismatch"):
        acc.image_metrics(np.zeros((2, 3, 3)), np.zeros((3, 2, 3)))


@pytest.mark.gpu
def test_gpu_reference_regression_chain(regression, tmp_path):
    """The reference's small regression end to end on the GPU: the analytic
    torus snapshot -> precompute_coefficient_bricks -> render_stokes_image_bricks
    against render_stokes_image, each stage against the reference's own output,
    and the reference's acceptance bounds (mean_abs <= 0.95, max_abs <= 1)."""
    from blackhole_native import accelerated as acc
    from blackhole_native import grrt, synchrotron

    g = regression
    snap, scaling = _reg_inputs(g)
    bricks = synchrotron.precompute_coefficient_bricks(snap, scaling, nu_hz=230e9, dtype="float32", stride=1)
    ref_b = g["brick_coeffs"].astype(np.float64)
    scale = np.maximum(np.abs(ref_b).max(axis=(0, 1, 2)), 1e-300)
    assert np.all(np.abs(bricks.coeffs - ref_b) <= 1e-6 * scale)
    ref = grrt.render_stokes_image(grrt.PolarizedRenderConfig(width=3, height=2, max_steps=40, step=0.18), snap, scaling)
    for py in range(2):
        for px in range(3):
            assert _rel(ref[py, px], g["reg_ref"][py, px]) <= 1e-10, (px, py)
    cand_cfg = acc.AcceleratedRenderConfig(width=3, height=2, max_steps=40, step=0.18, progressive_min_width=2)
    cand = acc.render_stokes_image_bricks(cand_cfg, snap, bricks)
    for py in range(2):
        for px in range(3):
            assert _rel(cand[py, px], g["reg_cand"][py, px]) <= TOL, (px, py)
    reg = acc.compare_reference_vs_bricks(ref, cand)
    assert np.isfinite(reg.metrics.mean_abs) and reg.metrics.mean_abs <= 0.95 and reg.metrics.max_abs <= 1.0
    assert np.allclose([reg.metrics.max_abs, reg.metrics.mean_abs], g["reg_metrics"][:2], rtol=0, atol=1e-6)

    frames = acc.render_progressive_stokes_bricks(
        acc.AcceleratedRenderConfig(width=8, height=6, max_steps=30, step=0.2, progressive_min_width=2), snap, bricks)
    assert np.array_equal(np.array([[f.level, f.width, f.height] for f in frames]), g["prog_levels"])
    for i, f in enumerate(frames):
        want = g[f"prog_{i}"]
        assert f.stokes.shape == want.shape
        for idx in np.ndindex(want.shape[:2]):
            assert _rel(f.stokes[idx], want[idx]) <= TOL if np.any(want[idx]) else not np.any(f.stokes[idx])
    acc.save_progressive_npz(frames[-1], tmp_path / "f.npz")
    with np.load(tmp_path / "f.npz") as z:
        assert z["stokes"].shape == (6, 8, 4)

    grid = SimpleNamespace(r=g["brick_r"], theta=g["brick_theta"], phi=g["brick_phi"], coeffs=g["brick_coeffs"])
    c = acc.sample_coefficient_brick(grid, *g["sample_point"])
    assert c is not None and c.shape == (11,) and _rel(c, g["sample_value"]) <= TOL
    assert acc.sample_coefficient_brick(grid, 1.0e3, 1.0, 1.0) is None


def _default_scene_view(stride_w=160, stride_h=90):
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = 0.9375, 55.0, np.radians(65.0), 0.0
    v.fov_y_deg, v.roll_deg, v.width, v.height = 32.0, 0.0, stride_w, stride_h
    return v


def _outbound_cases(golden):
    """(view, step, max_steps, r_edge, pixels): the golden scene, and every
    fourth row and column of the reference's default 160 x 90 image through
    the 40 M torus brick."""
    from blackhole_native import bricks

    cam = golden["acc_cam"]
    v = O.View()
    v.spin_a, v.r_obs, v.theta_obs, v.phi_obs = 0.9375, cam[0], cam[1], cam[2]
    v.fov_y_deg, v.roll_deg, v.width, v.height = cam[3], 0.0, 24, 16
    yield v, 0.1, 900, float(_grids(golden)[0].max()), [(x, y) for y in range(16) for x in range(24)]
    r_edge = float(np.asarray(bricks.torus_grids(128, 64, 128, 0.9375)[0], dtype=np.float32).max())
    yield _default_scene_view(), 0.06, 5000, r_edge, [(x, y) for y in range(0, 90, 4) for x in range(0, 160, 4)]


def test_outbound_exit_rule_on_full_oracle_traces(golden):
    """The brick renderer ends a ray once it is past the brick's outer radius
    moving out with R(r') >= E^2 r'^4 / 4 ahead (oracle.bricktrace.outbound_for_good
    restates the kernel's test).  On full oracle traces of both scenes no
    state after the first one the rule accepts lies at or inside the brick's
    outer radius or has r falling, so no later segment could have been
    sampled; the rule fires on most rays and shortens the longest trace."""
    for v, h, max_steps, r_edge, pixels in _outbound_cases(golden):
        full, cut, fired = [], [], 0
        for px, py in pixels:
            y0, pt, pphi = O.camera_ray(v, 2.0 * (px + 0.5) / v.width - 1.0, 1.0 - 2.0 * (py + 0.5) / v.height,
                                        v.width / v.height)
            st, _ = O.trace_rk4(y0, pt, pphi, v.spin_a, h, max_steps, 220.0)
            fire = B.outbound_for_good(st[1:], pt, pphi, v.spin_a, r_edge)
            k = int(np.argmax(fire)) + 1 if fire.any() else len(st) - 1
            fired += bool(fire.any())
            rest = st[k:, 1]
            assert not np.any(rest[1:] <= r_edge) and not np.any(np.diff(rest) <= 0.0), (px, py, k)
            full.append(len(st) - 1)
            cut.append(k)
        assert fired >= len(pixels) // 2
        assert max(cut) < max(full)
    # the default scene's longest trace: 4,798 steps in full, 1,734 to the exit (every fourth pixel)
    assert max(cut) < 0.5 * max(full)


def test_outbound_rule_declines_inbound_inside_and_near_periapsis():
    """Equatorial photons (p_theta = 0, E = 1) at r = 50 past a 40 M brick:
    the rule accepts an outward ray of small impact parameter and declines an
    inward one, one inside the brick, and an outward ray just past its
    periapsis (L = 48 ~ r), where R(r') >= E^2 r'^4 / 4 does not hold yet --
    such a ray escapes too, but the rule waits until the margin does."""
    a, E = 0.9375, 1.0
    r, th = 50.0, np.pi / 2
    # L chosen so that R(r) is small but positive at r (near a turning point) and dr/dlambda > 0
    for L, pr_sign, r0, want in ((3.0, 1.0, r, True), (3.0, -1.0, r, False), (3.0, 1.0, 30.0, False),
                                 (48.0, 1.0, r, False)):
        u, a2 = r0 * r0, a * a
        dlt = u - 2.0 * r0 + a2
        K = (L - a * E) ** 2  # p_theta = 0 on the equator
        R = (E * (u + a2) - a * L) ** 2 - dlt * K
        pr = pr_sign * np.sqrt(max(R, 0.0)) / dlt
        st = np.array([[0.0, r0, th, 0.0, pr, 0.0]])
        assert bool(B.outbound_for_good(st, -E, L, a, 40.0)[0]) is want, (L, pr_sign, r0)


@pytest.mark.gpu
def test_gpu_outbound_exit_keeps_the_image(golden):
    """The early exit changes no pixel: bit-identical images, optical depths
    and sampled-segment counts against full traces (full_trace=True), on the
    golden scene (with and without the optical-depth cutoff) and on the
    reference's default 160 x 90 image of the seeded 128 x 64 x 128 torus
    brick; rays ended outbound are ones the full trace ends as escaped or at
    max_steps, after no more steps."""
    import torch

    from blackhole_native import accelerated as acc
    from blackhole_native import bricks

    snap = SimpleNamespace(spin_a=0.9375)
    b = bricks.torus_brick(128, 64, 128, spin_a=0.9375, seed=0, dtype=np.float32)
    scenes = [(_config(acc, golden["acc_cam"], "rk2", cut), _golden_bricks(golden)) for cut in ("full", "cut")]
    scenes.append((acc.AcceleratedRenderConfig(), SimpleNamespace(r=b.r, theta=b.theta, phi=b.phi, coeffs=b.coeffs)))
    outbound = 0
    for cfg, grid in scenes:
        db = acc.DeviceBricks(grid)
        img, diag = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True)
        ref, rdiag = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True, full_trace=True)
        assert torch.equal(img, ref)
        assert torch.equal(diag[..., :2], rdiag[..., :2])
        st, rst = diag[..., 3].cpu().numpy(), rdiag[..., 3].cpu().numpy()
        out = st == 5  # BHN_RAY_OUTBOUND
        assert np.all(st[~out] == rst[~out]) and np.all(np.isin(rst[out], (0, 2)))
        assert torch.all(diag[..., 2] <= rdiag[..., 2]) and not np.any(rst == 5)
        outbound += int(out.sum())
    assert outbound > 0.5 * 160 * 90


@pytest.mark.gpu
def test_gpu_coefficient_layouts_give_one_image(golden):
    """The brick as the reference holds it ([..][11] float64) and as 12-wide
    cell records in float32 and float64 give bit-identical images and
    diagnostics: the records only change how the corners are loaded."""
    import torch

    from blackhole_native import accelerated as acc

    snap = SimpleNamespace(spin_a=0.9375)
    cfg = _config(acc, golden["acc_cam"], "rk2", "full")
    cfg = acc.AcceleratedRenderConfig(width=24, height=16, camera=cfg.camera, step=0.1, max_steps=900,
                                      transfer=cfg.transfer)
    db = acc.DeviceBricks(_golden_bricks(golden, np.float32))
    assert db.layout == acc.BRICK_F32X12 and db.records.shape[-1] == 12 and db.records.data_ptr() % 16 == 0
    ref = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True)
    wide = db.records[..., :11].to(torch.float64).contiguous()
    for layout, rec in ((acc.BRICK_F64X11, wide),
                        (acc.BRICK_F64X12, torch.nn.functional.pad(wide, (0, 1)).contiguous())):
        db.records, db.layout = rec, layout
        got = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True)
        assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1]), layout
    d64 = acc.DeviceBricks(_golden_bricks(golden, np.float64))
    assert d64.layout == acc.BRICK_F64X12


@pytest.mark.gpu
def test_gpu_one_and_two_warp_forms_agree(golden):
    """An image with more ray warps than 4 per SM runs the one-warp kernel; its
    tiles, small enough for the two-warp form (geodesic warp + transfer warp
    per 32 rays), must give the same pixels and diagnostics bit for bit."""
    import torch

    from blackhole_native import accelerated as acc
    from blackhole_native.tiles import RenderTile

    snap = SimpleNamespace(spin_a=0.9375)
    base = _config(acc, golden["acc_cam"], "rk2", "cut")
    cfg = acc.AcceleratedRenderConfig(width=256, height=160, camera=base.camera, step=0.1, max_steps=900,
                                      transfer=base.transfer)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert 256 * 160 // 32 > 4 * sms and 128 * 80 // 32 <= 4 * sms
    db = acc.DeviceBricks(_golden_bricks(golden))
    img, diag = acc.render_stokes_image_bricks_device(cfg, snap, db, diagnostics=True)
    for y0 in (0, 80):
        for x0 in (0, 128):
            t = RenderTile(level=0, y0=y0, x0=x0, x1=x0 + 128, y1=y0 + 80)
            ti, td = acc.render_stokes_image_bricks_device(cfg, snap, db, tile=t, diagnostics=True)
            assert torch.equal(ti, img[y0:y0 + 80, x0:x0 + 128]), (x0, y0)
            assert torch.equal(td, diag[y0:y0 + 80, x0:x0 + 128]), (x0, y0)
    st = diag[..., 3].cpu().numpy()
    assert np.any(st == 4) and np.any(st == 5)  # the cutoff and the outbound exit both occur
