"""The exact constant-coefficient Stokes step (polarized_transfer.py:51-70):
the oracle restatement (oracle/transfer.py) and the GPU micro-kernel
(bhn_stokes_exact_brick) against the reference's own stokes_step_exact
outputs (tests/golden/exact_step.npz, scipy.linalg.expm)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import transfer as T


@pytest.fixture(scope="module")
def golden():
    with np.load(Path(__file__).parent / "golden" / "exact_step.npz") as z:
        return {k: z[k] for k in z}


def _rel(got, ref):
    return float(np.max(np.abs(got - ref)) / max(float(np.max(np.abs(ref))), 1e-300))


def test_oracle_matches_reference(golden):
    for i, ds in enumerate(golden["exact_ds"]):
        for k, c in enumerate(golden["exact_coeffs"]):
            got = T.stokes_step_exact(golden["exact_initial"][k], c, float(ds))
            assert _rel(got, golden["exact_out"][i, k]) <= 1e-11, (i, k)


def test_oracle_limits():
    """Zero step is the identity; pure absorption decays as exp(-alpha ds);
    the steady state is K^-1 j."""
    c = np.zeros(11)
    c[:4] = [1.0, 0.2, 0.1, 0.0]
    c[4] = 2.0
    S0 = np.array([0.3, -0.1, 0.05, 0.01])
    assert np.array_equal(T.stokes_step_exact(S0, c, 0.0), S0)
    want = S0 * np.exp(-2.0 * 0.7) + c[:4] / 2.0 * (1.0 - np.exp(-2.0 * 0.7))
    np.testing.assert_allclose(T.stokes_step_exact(S0, c, 0.7), want, rtol=1e-13)
    c2 = np.array([1.0, 0.5, 0.2, 0.1, 3.0, 1.0, -0.5, 0.3, 5.0, -2.0, 1.0])
    steady = np.linalg.solve(T.propagation_matrix(c2), c2[:4])
    np.testing.assert_allclose(T.stokes_step_exact(S0, c2, 500.0), steady, rtol=1e-10)


@pytest.mark.gpu
def test_gpu_exact_step_matches_reference(golden):
    import blackhole_native as bn

    coeffs = golden["exact_coeffs"]
    for i, ds in enumerate(golden["exact_ds"]):
        out = np.asarray(bn.stokes_exact_brick(coeffs.reshape(-1).tolist(), float(ds),
                                               golden["exact_initial"].reshape(-1).tolist())).reshape(-1, 4)
        for k in range(coeffs.shape[0]):
            assert _rel(out[k], golden["exact_out"][i, k]) <= 1e-11, (i, k)
    # broadcast initial, device tensors in, device tensor out
    import torch

    dc = torch.as_tensor(coeffs, device="cuda")
    res = bn.stokes_exact_brick(dc, 0.1, torch.as_tensor([1.0, 0.0, 0.0, 0.0], device="cuda"))
    assert res.is_cuda and res.numel() == 4 * coeffs.shape[0]
    want = np.array([T.stokes_step_exact([1.0, 0.0, 0.0, 0.0], c, 0.1) for c in coeffs])
    assert _rel(res.cpu().numpy().reshape(-1, 4), want) <= 1e-11


@pytest.mark.gpu
def test_gpu_exact_step_rejects_like_rk2():
    import blackhole_native as bn

    with pytest.raises(ValueError, match="ds_cm must be finite and non-negative"):
        bn.stokes_exact_brick([1.0] * 11, -1.0, [0.0] * 4)
    with pytest.raises(ValueError, match="initial must contain"):
        bn.stokes_exact_brick([1.0] * 22, 0.1, [0.0] * 5)
    with pytest.raises(ValueError, match="11-coefficient"):
        bn.stokes_exact_brick([1.0] * 10, 0.1, [0.0] * 4)
