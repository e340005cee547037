"""Host-side logic: argument validation (reference messages), views, the
synthetic torus brick."""

from __future__ import annotations

import math

import numpy as np
import pytest

import blackhole_native as bn
from blackhole_native import bricks
from tests.helpers import linear_coeff_fixture


# -- argument validation happens before any device work (native/core/src/lib.rs:112-169, 229-255, 318-334)
def test_stokes_rk2_brick_validation_messages():
    with pytest.raises(ValueError, match="ds_cm must be finite and non-negative"):
        bn.stokes_rk2_brick([0.0] * 11, -1.0, [0.0] * 4)
    with pytest.raises(ValueError, match="ds_cm must be finite and non-negative"):
        bn.stokes_rk2_brick([0.0] * 11, float("nan"), [0.0] * 4)
    with pytest.raises(ValueError, match="one or more flat 11-coefficient cells"):
        bn.stokes_rk2_brick([0.0] * 10, 0.1, [0.0] * 4)
    with pytest.raises(ValueError, match="one or more flat 11-coefficient cells"):
        bn.stokes_rk2_brick([], 0.1, [0.0] * 4)
    with pytest.raises(ValueError, match="coeffs must contain only finite values"):
        bn.stokes_rk2_brick([float("inf")] + [0.0] * 10, 0.1, [0.0] * 4)
    with pytest.raises(ValueError, match="initial must contain either 4 values or 4 values per coefficient cell"):
        bn.stokes_rk2_brick([0.0] * 22, 0.1, [0.0] * 5)
    with pytest.raises(ValueError, match="initial must contain only finite values"):
        bn.stokes_rk2_brick([0.0] * 11, 0.1, [float("nan"), 0, 0, 0])


def test_sampler_validation_messages():
    c, rg, tg, pg = linear_coeff_fixture()
    flat = c.ravel()
    with pytest.raises(ValueError, match="r grid must contain at least 2 values"):
        bn.sample_brick_trilinear(flat, [0.0], tg, pg, [0.5, 0.5, 0.5])
    with pytest.raises(ValueError, match="theta grid must contain only finite values"):
        bn.sample_brick_trilinear(flat, rg, [0.0, float("nan")], pg, [0.5, 0.5, 0.5])
    with pytest.raises(ValueError, match="phi grid must be strictly increasing"):
        bn.sample_brick_trilinear(flat, rg, tg, [1.0, 1.0], [0.5, 0.5, 0.5])
    with pytest.raises(ValueError, match="coeffs must contain exactly r\\*theta\\*phi\\*11 values; expected 88, got 87"):
        bn.sample_brick_trilinear(flat[:-1], rg, tg, pg, [0.5, 0.5, 0.5])
    with pytest.raises(ValueError, match="points must contain flat r, theta, phi triples"):
        bn.sample_brick_trilinear(flat, rg, tg, pg, [0.5, 0.5])
    with pytest.raises(ValueError, match="points must contain only finite values"):
        bn.sample_brick_trilinear(flat, rg, tg, pg, [0.5, float("inf"), 0.5])
    with pytest.raises(ValueError, match="initial must contain either 4 values or 4 values per sample point"):
        bn.sample_and_step_stokes(flat, rg, tg, pg, [0.5, 0.5, 0.5], 0.1, [0.0] * 8)
    with pytest.raises(ValueError, match="invalid_policy"):
        bn.sample_and_step_stokes(flat, rg, tg, pg, [0.5, 0.5, 0.5], 0.1, [0.0] * 4, invalid_policy="break")
    with pytest.raises(ValueError, match="ds_cm must be finite and non-negative"):
        bn.sample_and_step_stokes(flat, rg, tg, pg, [0.5, 0.5, 0.5], -0.1, [0.0] * 4)


def test_view_validation():
    bn.View(32, 18).validate()
    with pytest.raises(ValueError, match="outer horizon"):
        bn.View(8, 8, r_obs=1.2, spin_a=0.5).validate()
    with pytest.raises(ValueError, match="pole"):
        bn.View(8, 8, inclination_deg=0.0).validate()
    with pytest.raises(ValueError, match="crop"):
        bn.View(8, 8, crop=(4, 4, 8, 8)).validate()
    with pytest.raises(ValueError, match="Kerr spin"):
        bn.View(8, 8, spin_a=1.0).validate()
    s = bn.View(1024, 1024, crop=(480, 480, 64, 64)).to_struct(123)
    assert (s.x0, s.y0, s.crop_w, s.crop_h, s.out_offset) == (480, 480, 64, 64, 123)
    assert abs(s.fov_y_deg - 2.0 * math.degrees(math.atan(0.02))) < 1e-12


def test_torus_brick_is_seeded_and_follows_the_formula():
    a = bricks.torus_brick(6, 5, 4, spin_a=0.9375, seed=3, dtype=np.float64)
    b = bricks.torus_brick(6, 5, 4, spin_a=0.9375, seed=3, dtype=np.float64)
    c = bricks.torus_brick(6, 5, 4, spin_a=0.9375, seed=4, dtype=np.float64)
    assert np.array_equal(a.coeffs, b.coeffs) and not np.array_equal(a.coeffs, c.coeffs)
    rp = 1.0 + math.sqrt(1.0 - 0.9375 ** 2)
    assert abs(a.r[0] - 1.05 * rp) < 1e-12 and abs(a.r[-1] - 40.0) < 1e-12
    np.testing.assert_allclose(np.diff(np.log(a.r)), np.log(40.0 / (1.05 * rp)) / 5, rtol=1e-10)
    np.testing.assert_allclose(a.theta, math.pi * (np.arange(5) + 0.5) / 5)
    np.testing.assert_allclose(a.phi, np.arange(4) * 2 * math.pi / 4)
    dens = np.exp(-((a.r[:, None, None] - 8.0) ** 2) / 8.0 - 4.0 * np.cos(a.theta)[None, :, None] ** 2)
    ratio = a.coeffs[..., 0] / dens
    assert np.all(np.abs(np.log(ratio)) < 6 * bricks.LOGNORMAL_SIGMA)     # lognormal noise only
    np.testing.assert_array_less(a.coeffs[..., 4] / a.coeffs[..., 0], 0.1 * np.exp(6 * bricks.LOGNORMAL_SIGMA))
    assert np.all(a.coeffs[..., 8] / dens <= bricks.ROTATIVITY_SCALES[0] * 1.5 * np.exp(6 * bricks.LOGNORMAL_SIGMA))
    f32 = bricks.torus_brick(6, 5, 4, spin_a=0.9375, seed=3, dtype=np.float32)
    assert f32.coeffs.dtype == np.float32
    assert np.array_equal(f32.r.astype(np.float32).astype(np.float64), f32.r)


def test_brick_grid_validation():
    with pytest.raises(ValueError, match="strictly increasing"):
        bn.BrickGrid([0.0, 0.0], [0.0, 1.0], [0.0, 1.0], np.zeros((2, 2, 2, 11)))
    with pytest.raises(ValueError, match="coeffs must have shape"):
        bn.BrickGrid([0.0, 1.0], [0.0, 1.0], [0.0, 1.0], np.zeros((2, 2, 3, 11)))


def test_brick_npz_round_trip(tmp_path):
    a = bricks.torus_brick(4, 3, 5, spin_a=0.5, seed=1, dtype=np.float32)
    a.save_npz(tmp_path / "b.npz")
    b = bn.BrickGrid.load_npz(tmp_path / "b.npz")
    assert np.array_equal(a.coeffs, b.coeffs) and np.array_equal(a.r, b.r) and b.spin_a == 0.5


def test_render_prepare_rejects_outputs_beyond_32_bit_indices():
    """The kernels keep a ray's output index in 32 bits: bhn_render_prepare
    refuses views whose packed outputs reach past 2^32 pixels (checked on the
    host, before any device work)."""
    import ctypes

    from blackhole_native import _lib

    L = _lib.lib()
    L.bhn_render_prepare.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    L.bhn_render_prepare.restype = ctypes.c_int
    v = bn.View(1024, 1024).to_struct((1 << 32) - 1024 * 1024 + 1)
    scratch = ctypes.create_string_buffer((1 << 16) + 256)
    aligned = (ctypes.addressof(scratch) + 255) & ~255
    rc = L.bhn_render_prepare(ctypes.byref(v), 1, aligned, 1 << 16, None)
    assert rc == 1 and b"2^32" in L.bhn_last_error()


def test_estimate_brick_memory_and_float16_bricks(tmp_path):
    """coefficient_bricks.py:155-160 and float16 CoefficientBrickGrid values
    (kept as float16, through the npz round trip)."""
    est = bn.estimate_brick_memory(8, 6, 4, "float32")
    assert est["coeff_bytes"] == 8 * 6 * 4 * 11 * 4 and est["grid_bytes"] == 18 * 4
    assert est["total_bytes"] == est["coeff_bytes"] + est["grid_bytes"] > 8 * 6 * 4 * 11 * 3
    assert est["total_mib"] == est["total_bytes"] / (1024.0 * 1024.0)
    assert bn.estimate_brick_memory(8, 6, 4, "float16")["coeff_bytes"] == 8 * 6 * 4 * 11 * 2
    b = bricks.torus_brick(5, 4, 3, spin_a=0.5, seed=2, dtype=np.float32)
    h = bn.BrickGrid(b.r, b.theta, b.phi, b.coeffs.astype(np.float16), spin_a=0.5, nu_hz=86e9)
    assert h.coeffs.dtype == np.float16
    h.save_npz(tmp_path / "h.npz")
    back = bn.BrickGrid.load_npz(tmp_path / "h.npz")
    assert back.coeffs.dtype == np.float16 and np.array_equal(back.coeffs, h.coeffs) and back.nu_hz == 86e9


def test_brick_grid_reports_dtype_and_bytes():
    b = bricks.torus_brick(5, 4, 3, spin_a=0.5, seed=2, dtype=np.float32)
    assert b.dtype_name == "float32" and b.bytes == b.coeffs.nbytes + 4 * (5 + 4 + 3)
    est = bn.estimate_brick_memory(5, 4, 3, "float32")
    assert b.bytes == est["total_bytes"]
