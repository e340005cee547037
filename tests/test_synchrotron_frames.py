"""Per-frame synchrotron coefficients: ThermalSynchrotronCoefficients,
NonthermalPowerLawSynchrotronCoefficients and HybridSynchrotronCoefficients
``.coefficients(frame, nu_hz)`` (python/blackhole_sim/synchrotron.py:248, 290,
318).  CPU: the oracle against fixtures the reference's own models wrote
(tests/golden/synchrotron_frames.npz).  GPU: ``bhn_synchrotron_coefficients``
(through the package's batch and single-frame calls) against the same
fixtures, to 1e-12 of each channel's largest magnitude."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import synchrotron as S

GOLDEN = Path(__file__).parent / "golden" / "synchrotron_frames.npz"
MODELS = {
    "hybrid": (dict(S.THERMAL), dict(S.NONTHERMAL)),
    "thermal": (dict(gamma_grid_size=96, pitch_nodes=9, faraday_rotation_scale=0.7, faraday_conversion_scale=1.3),
                None),
    "nonthermal": (None, dict(p=2.8, gamma_min=30.0, gamma_max=3e4, nonthermal_fraction=0.1, gamma_grid_size=100,
                              pitch_nodes=12, absorption_scale=0.5, faraday_scale=0.3)),
    "hybrid_custom": (dict(S.THERMAL, gamma_grid_size=64, pitch_nodes=8),
                      dict(S.NONTHERMAL, gamma_grid_size=300, pitch_nodes=20)),
}
CASES = [(name, nu) for name in MODELS for nu in (230e9, 86e9)]


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z}


def _err(out, ref):
    """Largest error relative to each channel's largest magnitude."""
    scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    return float(np.max(np.abs(out - ref) / scale))


def _oracle(frames, th, nt, nu):
    out = np.zeros((len(frames), 11))
    for i, (n_e, te, b, cos_los, chi) in enumerate(frames):
        if th is not None:
            out[i] += S.thermal(n_e, te, b, chi, nu, th, cos_los=cos_los)
        if nt is not None:
            out[i] += S.nonthermal(n_e, te, b, chi, nu, nt, cos_los=cos_los)
    return out


@pytest.mark.parametrize("name,nu", CASES)
def test_oracle_matches_reference_frames(golden, name, nu):
    ref = golden[f"{name}_{int(nu / 1e9)}"]
    out = _oracle(golden["frames"], *MODELS[name], nu)
    assert np.array_equal(out == 0.0, ref == 0.0)
    assert _err(out, ref) <= 1e-12


def _model(name):
    import blackhole_native as bn

    th, nt = MODELS[name]
    T = bn.ThermalSynchrotronCoefficients(**th) if th else None
    N = bn.NonthermalPowerLawSynchrotronCoefficients(**nt) if nt else None
    if T is not None and N is not None:
        return bn.HybridSynchrotronCoefficients(T, N)
    return T if T is not None else N


def test_kernel_table_first_guess_is_within_one_segment():
    """The device lookup of the F / G table takes the segment guess
    (lx - lx[0]) * inv and corrects it by at most one knot each way.  That is
    exact when the guess is never off by more than one, which holds for the
    table's log-uniform knots (log of the geomspace(1e-8, 1e3, 256) built like
    the device table): checked at the knots, their float neighbours and a
    million random points against numpy's searchsorted (numpy.interp's
    segment)."""
    n = 256
    ls, le = np.log10(1.0e-8), np.log10(1.0e3)
    step = (le - ls) / (n - 1)
    x = 10.0 ** (np.arange(n) * step + ls)
    x[0], x[-1] = 1.0e-8, 1.0e3
    lx = np.log(x)
    inv = (n - 1) / (lx[-1] - lx[0])
    rng = np.random.default_rng(7)
    pts = np.concatenate([lx, np.nextafter(lx, -np.inf), np.nextafter(lx, np.inf),
                          rng.uniform(lx[0], lx[-1], 1_000_000)])
    pts = np.clip(pts, lx[0], lx[-1])
    guess = np.clip(((pts - lx[0]) * inv).astype(np.int64), 0, n - 2)
    true = np.clip(np.searchsorted(lx, pts, side="right") - 1, 0, n - 2)
    assert np.abs(guess - true).max() <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("name,nu", CASES)
def test_gpu_frames_match_reference(golden, name, nu):
    ref = golden[f"{name}_{int(nu / 1e9)}"]
    model = _model(name)
    got = model.coefficients_batch(golden["frames"], nu)
    assert got.shape == ref.shape and got.dtype == np.float64
    # exact zeros agree, except where the reference's value is only the sum of
    # its kernel table's floored tail (F, G = 1e-300 beyond x = 1e3: denormals
    # of 1e-321 .. 1e-312 for cold, weakly magnetised frames), which the kernel
    # leaves out and returns as 0
    differ = (got == 0.0) != (ref == 0.0)
    assert np.all(np.abs(ref[differ]) < 1e-290) and np.all(np.abs(got[differ]) < 1e-290)
    assert _err(got, ref) <= 1e-12
    nz = np.abs(ref) >= 1e-290
    assert np.max(np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])) <= 1e-11


@pytest.mark.gpu
def test_gpu_frame_objects_and_device_tensors(golden):
    import blackhole_native as bn

    model = bn.HybridSynchrotronCoefficients()
    frames = golden["frames"]
    ref = golden["hybrid_230"]
    one = model.coefficients(bn.LocalPlasmaFrame(*frames[3].tolist()), 230e9)
    assert isinstance(one, bn.PolarizedCoefficients)
    np.testing.assert_allclose(one.as_array(), ref[3], rtol=1e-11, atol=1e-12 * np.abs(ref).max(axis=0).max())
    objs = [bn.LocalPlasmaFrame(*f.tolist()) for f in frames[:5]]
    assert np.array_equal(model.coefficients_batch(objs, 230e9), model.coefficients_batch(frames[:5], 230e9))
    dev_out = model.coefficients_batch(torch.from_numpy(frames).cuda(), 230e9)
    assert dev_out.is_cuda and np.array_equal(dev_out.cpu().numpy(), model.coefficients_batch(frames, 230e9))
    K = one.propagation_matrix()
    assert K.shape == (4, 4) and np.allclose(np.diag(K), one.alpha_i)
    with pytest.raises(ValueError, match="frames"):
        model.coefficients_batch(np.zeros((3, 4)), 230e9)
