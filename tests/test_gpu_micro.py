"""GPU parity of the plugin micro-kernels (float64): bit-exact against the
reference's own outputs (golden vectors) and the oracle."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import blackhole_native as bn
from oracle import oracle as O
from tests.helpers import linear_coeff_fixture, rust_linear_fixture

pytestmark = pytest.mark.gpu

PREFIXES = ("fix4", "bench", "rand")
DS = {"fix4": 0.05, "bench": 0.05, "rand": 0.37}


def _args(g, pre):
    return (g[f"{pre}_coeffs"].ravel(), g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_phi"], g[f"{pre}_points"].ravel())


def _initial(g, pre):
    return g[f"{pre}_initial"] if f"{pre}_initial" in g else np.array([1e-2, 1e-3, 0.0, 0.0])


@pytest.mark.parametrize("pre", PREFIXES)
def test_sample_brick_trilinear_bit_exact(micro_golden, pre):
    g = micro_golden
    out = np.asarray(bn.sample_brick_trilinear(*_args(g, pre))).reshape(-1, 11)
    assert np.array_equal(out, g[f"{pre}_sample"], equal_nan=True)
    # device-tensor fast path
    dev = [torch.as_tensor(x, device="cuda") for x in _args(g, pre)]
    outd = bn.sample_brick_trilinear(*dev).cpu().numpy().reshape(-1, 11)
    assert np.array_equal(outd, g[f"{pre}_sample"], equal_nan=True)


@pytest.mark.parametrize("pre", PREFIXES)
def test_sample_and_step_stokes_bit_exact(micro_golden, pre):
    g = micro_golden
    ini = _initial(g, pre)
    raw = np.asarray(bn.sample_and_step_stokes(*_args(g, pre), DS[pre], ini.ravel())).reshape(-1, 4)
    assert np.array_equal(raw, g[f"{pre}_step_nan"], equal_nan=True)
    # the reference wrapper applies the policy after the native call (native_kernels.py:391-397)
    valid = np.asarray(bn.sample_brick_valid_mask(g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_points"].ravel()))
    n = raw.shape[0]
    ini_b = np.broadcast_to(ini, (n, 4)) if ini.size == 4 else ini.reshape(n, 4)
    for pol in ("initial", "zero"):
        wrapped = raw.copy()
        wrapped[~valid] = ini_b[~valid] if pol == "initial" else 0.0
        assert np.array_equal(wrapped, g[f"{pre}_step_{pol}"], equal_nan=True)
        dev_pol = np.asarray(bn.sample_and_step_stokes(*_args(g, pre), DS[pre], ini.ravel(), invalid_policy=pol))
        assert np.array_equal(dev_pol.reshape(-1, 4), g[f"{pre}_step_{pol}"], equal_nan=True)


def test_valid_mask_bit_exact(micro_golden):
    g = micro_golden
    for pre in ("fix4", "rand"):
        m = np.asarray(bn.sample_brick_valid_mask(g[f"{pre}_r"], g[f"{pre}_theta"], g[f"{pre}_points"]))
        assert np.array_equal(m, g[f"{pre}_mask"])
        md = bn.sample_brick_valid_mask(*(torch.as_tensor(g[k], device="cuda")
                                          for k in (f"{pre}_r", f"{pre}_theta", f"{pre}_points")))
        assert np.array_equal(md.cpu().numpy(), g[f"{pre}_mask"])


def test_stokes_rk2_brick_bit_exact(micro_golden):
    g = micro_golden
    out = np.asarray(bn.stokes_rk2_brick(g["det_coeffs"].ravel(), 0.05, g["det_initial"].ravel()))
    assert np.array_equal(out.reshape(g["det_step"].shape), g["det_step"])
    out = np.asarray(bn.stokes_rk2_brick(g["det_coeffs"].ravel(), 0.3, [0.5, -0.1, 0.2, 0.05]))
    assert np.array_equal(out.reshape(g["det_step"].shape), g["det_step_broadcast"])
    out = bn.stokes_rk2_brick(torch.as_tensor(g["rand_rk2_coeffs"], device="cuda"), 0.11,
                              torch.as_tensor(g["rand_rk2_initial"], device="cuda"))
    assert np.array_equal(out.cpu().numpy().reshape(-1, 4), g["rand_rk2_step"])


def test_reference_known_answers_on_gpu():
    out = bn.stokes_rk2_brick([1.0, 0, 0, 0, 0.5, 0, 0, 0, 0, 0, 0], 0.1, [0.0, 0.0, 0.0, 0.0])
    assert abs(out[0] - 0.0975) < 1e-12 and out[1:] == [0.0, 0.0, 0.0]
    s = bn.sample_brick_trilinear(rust_linear_fixture(), [0.0, 1.0], [0.0, 1.0], [0.0, 1.0], [0.5, 0.5, 0.5])
    assert len(s) == 11 and abs(s[0] - 55.5) < 1e-12 and abs(s[10] - 55.51) < 1e-12
    s = bn.sample_brick_trilinear(rust_linear_fixture(), [0.0, 1.0], [0.0, 1.0], [0.0, 1.0],
                                  [-0.1, 0.5, 0.5, 0.5, 1.1, 0.5])
    assert len(s) == 22 and all(math.isnan(x) for x in s)
    s = bn.sample_and_step_stokes(rust_linear_fixture(), [0.0, 1.0], [0.0, 1.0], [0.0, 1.0], [-0.1, 0.5, 0.5], 0.1,
                                  [1.0, 2.0, 3.0, 4.0])
    assert len(s) == 4 and all(math.isnan(x) for x in s)
    c, rg, tg, pg = linear_coeff_fixture()
    s = np.asarray(bn.sample_brick_trilinear(c.ravel(), rg, tg, pg, [0.25, 0.5, 0.75]))
    np.testing.assert_allclose(s, 30.75 + np.arange(11) * 0.125, rtol=1e-12, atol=1e-12)


def test_empty_inputs():
    c, rg, tg, pg = linear_coeff_fixture()
    assert bn.sample_brick_trilinear(c.ravel(), rg, tg, pg, []) == []
    assert bn.sample_and_step_stokes(c.ravel(), rg, tg, pg, [], 0.1, [0.0] * 4) == []
    assert bn.sample_brick_valid_mask(rg, tg, []) == []


def test_large_random_batch_bit_exact():
    """One million points on an irregular 33x17x29 grid: the GPU equals the oracle bit for bit."""
    rng = np.random.default_rng(5)
    rg = np.cumsum(rng.uniform(0.05, 1.0, 33))
    tg = np.cumsum(rng.uniform(0.01, 0.2, 17))
    pg = np.sort(rng.uniform(0, 2 * np.pi, 29))
    c = rng.normal(size=(33, 17, 29, 11))
    n = 1_000_000
    pts = np.stack([rng.uniform(rg[0] - 0.5, rg[-1] + 0.5, n), rng.uniform(tg[0] - 0.1, tg[-1] + 0.1, n),
                    rng.uniform(-50, 50, n)], axis=1)
    pts[:1000, 0] = rg[rng.integers(0, 33, 1000)]          # exact knots
    pts[1000:2000, 1] = tg[rng.integers(0, 17, 1000)]
    pts[2000:3000, 2] = pg[rng.integers(0, 29, 1000)] + 2 * np.pi * rng.integers(-5, 6, 1000)
    ini = rng.normal(size=(n, 4))
    dc, drg, dtg, dpg, dpts, dini = (torch.as_tensor(x, device="cuda") for x in (c, rg, tg, pg, pts, ini))
    got = bn.sample_brick_trilinear(dc, drg, dtg, dpg, dpts).cpu().numpy().reshape(n, 11)
    assert np.array_equal(got, O.sample_brick_trilinear(c, rg, tg, pg, pts), equal_nan=True)
    got = bn.sample_and_step_stokes(dc, drg, dtg, dpg, dpts, 0.21, dini, invalid_policy="initial")
    want = O.sample_and_step_stokes(c, rg, tg, pg, pts, 0.21, ini, "initial")
    assert np.array_equal(got.cpu().numpy().reshape(n, 4), want, equal_nan=True)
    m = bn.sample_brick_valid_mask(drg, dtg, dpts).cpu().numpy()
    assert np.array_equal(m, O.sample_brick_valid_mask(rg, tg, pts))


def test_device_validation_messages():
    c, rg, tg, pg = linear_coeff_fixture()
    dc = torch.as_tensor(c.ravel(), device="cuda")
    bad_grid = torch.tensor([0.0, 0.0], device="cuda", dtype=torch.float64)
    with pytest.raises(ValueError, match="r grid must be strictly increasing"):
        bn.sample_brick_trilinear(dc, bad_grid, torch.as_tensor(tg, device="cuda"), torch.as_tensor(pg, device="cuda"),
                                  torch.tensor([0.5, 0.5, 0.5], device="cuda", dtype=torch.float64))
    dc2 = dc.clone()
    dc2[3] = float("nan")
    with pytest.raises(ValueError, match="coeffs must contain only finite values"):
        bn.stokes_rk2_brick(dc2, 0.1, torch.zeros(4, device="cuda", dtype=torch.float64))


def test_throughput_probes_run_and_count():
    """The FP32 / FP64 throughput probes (roofline denominators) launch, report
    their operation counts and reject a bad mode."""
    import ctypes

    from blackhole_native import _lib

    L = _lib.lib()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    scratch = torch.empty(sms * 256 * 2, dtype=torch.float64, device="cuda")
    ops = ctypes.c_int64()
    _lib.check(L.bhn_fp32_peak_probe(scratch.data_ptr(), 2, 1, ctypes.byref(ops), None))
    assert ops.value == sms * 256 * 2 * 16 * 8 * 2
    _lib.check(L.bhn_fp64_peak_probe(scratch.data_ptr(), 2, 1, 0, ctypes.byref(ops), None))
    assert ops.value == sms * 256 * 2 * 16 * 8 * 2
    _lib.check(L.bhn_fp64_peak_probe(scratch.data_ptr(), 3, 1, 1, ctypes.byref(ops), None))
    assert ops.value == sms * 256 * 3 * 4 * 8
    torch.cuda.synchronize()
    assert L.bhn_fp64_peak_probe(scratch.data_ptr(), 2, 1, 2, ctypes.byref(ops), None) != 0
    assert b"probe mode" in L.bhn_last_error()


def test_cell_ordered_sampler_equals_the_plain_kernel():
    """bhn_sample_and_step_stokes_sorted and bhn_sample_brick_trilinear_sorted
    (points taken in brick-cell order, results written to their own rows) give
    the plain kernels' bits: every policy, broadcast and per-point initial
    vectors, points outside the domain, on knots and NaN points."""
    import torch

    from blackhole_native import _device as dev
    from blackhole_native import _lib, bricks, kernels

    b = bricks.torus_brick(24, 16, 20, spin_a=0.9, seed=3, dtype=np.float64)
    rng = np.random.default_rng(5)
    n = kernels.SORT_MIN_POINTS + 12345
    lo = [b.r[0] - 1.0, b.theta[0] - 0.1, -7.0]
    hi = [b.r[-1] + 1.0, b.theta[-1] + 0.1, 7.0]
    pts = rng.uniform(lo, hi, (n, 3))
    pts[::997] = np.nan
    pts[1::991, 0] = b.r[-1]
    pts[2::983, 1] = b.theta[0]
    pts[3::977, 2] = b.phi[0] + 2.0 * np.pi
    device = torch.device("cuda", 0)
    c = torch.as_tensor(b.coeffs.reshape(-1), device=device)
    rg, tg, pg = (torch.as_tensor(g, device=device) for g in (b.r, b.theta, b.phi))
    dp = torch.as_tensor(pts, device=device)
    L = _lib.lib()
    for per_point in (False, True):
        ini = torch.as_tensor(rng.normal(0.0, 1.0, 4 * n if per_point else 4), device=device)
        for policy in (0, 1, 2):
            plain = torch.empty(4 * n, dtype=torch.float64, device=device)
            _lib.check(L.bhn_sample_and_step_stokes(dev.ptr(c), dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(),
                                                    dev.ptr(pg), pg.numel(), dev.ptr(dp), n, 0.07, dev.ptr(ini),
                                                    ini.numel(), policy, dev.ptr(plain), dev.stream_ptr()))
            ordered = torch.empty_like(plain)
            kernels._launch_sample_and_step(c, rg, tg, pg, dp, n, 0.07, ini, policy, ordered)
            assert torch.equal(plain.view(torch.int64), ordered.view(torch.int64)), (per_point, policy)
    plain = torch.empty(11 * n, dtype=torch.float64, device=device)
    _lib.check(L.bhn_sample_brick_trilinear(dev.ptr(c), dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(), dev.ptr(pg),
                                            pg.numel(), dev.ptr(dp), n, dev.ptr(plain), dev.stream_ptr()))
    ordered = torch.empty_like(plain)
    kernels._launch_sample_trilinear(c, rg, tg, pg, dp, n, ordered)
    assert torch.equal(plain.view(torch.int64), ordered.view(torch.int64))
    plain = torch.empty(4 * n, dtype=torch.float64, device=device)
    assert L.bhn_sample_sort_scratch_bytes(n, b.cells) > 16 * n
    assert L.bhn_sample_sort_scratch_bytes(0, b.cells) == -1 and L.bhn_sample_sort_scratch_bytes(n, 0) == -1
    rc = L.bhn_sample_and_step_stokes_sorted(dev.ptr(c), dev.ptr(rg), rg.numel(), dev.ptr(tg), tg.numel(),
                                             dev.ptr(pg), pg.numel(), dev.ptr(dp), n, 0.07, dev.ptr(ini), ini.numel(),
                                             0, dev.ptr(plain), None, 0, dev.stream_ptr())
    assert rc == 1 and b"scratch" in L.bhn_last_error()
