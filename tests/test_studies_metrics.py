"""CPU checks of the study metrics (rel L1, capped rel L1, stability mask,
flux-weighted polarization-fraction error)."""

from __future__ import annotations

import numpy as np

from blackhole_native import studies


def _img(I, Q=0.0, U=0.0, V=0.0):
    I = np.asarray(I, dtype=np.float64)
    return np.stack([I, np.full_like(I, Q), np.full_like(I, U), np.full_like(I, V)], axis=-1)


def test_rel_l1_and_capped():
    b = np.array([1.0, 2.0, 3.0, 4.0])
    a = b.copy()
    a[1] = 1e30
    assert studies.rel_l1(b, b) == 0.0
    assert studies.rel_l1(a, b) > 1e28
    # the blown-up pixel counts as wholly wrong: |b_1| / sum |b|
    assert abs(studies.capped_rel_l1(a, b) - 2.0 / 10.0) < 1e-15
    a[2] = np.nan
    assert abs(studies.capped_rel_l1(a, b) - 5.0 / 10.0) < 1e-15


def test_stable_mask():
    ref = _img([1.0, 1.0, 2.0, -1.0, np.nan])
    p1 = _img([1.0 + 1e-6, 1.1, 2.0, -1.0, 1.0])
    p2 = _img([1.0, 1.0, np.inf, -1.0, 1.0])
    m = studies.stable_mask(ref, (p1, p2), scale=1.0)
    assert m.tolist() == [True, False, False, False, False]


def test_image_errors_and_dm():
    ref = _img([1.0, 2.0, 4.0], Q=0.1, U=0.0)
    img = _img([1.0, 2.0, 4.0], Q=0.1, U=0.0)
    img[2, 1] = 0.2  # m changes by 0.1 / 4 at the pixel of weight 4
    mask = np.ones(3, dtype=bool)
    e = studies.image_errors(img, ref, mask, scale=1.0)
    assert e["rel_l1_I"] == 0.0 and e["bad_frac"] == 0.0
    assert abs(e["rel_l1_Q"] - 0.1 / 0.3) < 1e-12
    assert abs(e["flux_weighted_dm"] - (4.0 * 0.025) / 7.0) < 1e-12
    assert studies.median_lit(np.array([0.0, 1.0, 3.0, np.nan])) == 2.0
