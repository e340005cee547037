"""Brick files interchangeable with the reference's CoefficientBrickGrid
(coefficient_bricks.py:57-75) and the tile / progressive-level helpers
(tiles.py:9-59), plus the GPU progressive renderer."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import blackhole_native as bn
from blackhole_native import tiles


def test_reads_reference_brick_file():
    b = bn.BrickGrid.load_npz(Path(__file__).parent / "golden" / "reference_brick.npz")
    assert b.coeffs.shape == (4, 3, 5, 11) and b.coeffs.dtype == np.float32
    assert b.nu_hz == 86e9 and b.spin_a == 0.5
    with np.load(Path(__file__).parent / "golden" / "reference_brick.npz") as z:
        assert np.array_equal(b.coeffs, z["coeffs"]) and np.array_equal(b.r, z["r"].astype(np.float64))


def test_writes_reference_layout(tmp_path):
    ref_keys = set(np.load(Path(__file__).parent / "golden" / "reference_brick.npz").files)
    b = bn.torus_brick(6, 4, 5, spin_a=0.3, seed=2)
    b.save_npz(tmp_path / "x" / "b.npz")
    with np.load(tmp_path / "x" / "b.npz") as z:
        assert set(z.files) == ref_keys
        assert str(z["dtype_name"]) == "float32" and float(z["nu_hz"]) == 230e9
    c = bn.BrickGrid.load_npz(tmp_path / "x" / "b.npz")
    assert np.array_equal(c.coeffs, b.coeffs) and c.spin_a == 0.3


def test_rejects_foreign_channel_order(tmp_path):
    b = bn.torus_brick(3, 3, 3, spin_a=0.3, seed=2)
    np.savez(tmp_path / "bad.npz", r=b.r, theta=b.theta, phi=b.phi, coeffs=b.coeffs,
             coeff_names=np.array(list(reversed(bn.COEFF_NAMES))))
    with pytest.raises(ValueError, match="channels"):
        bn.BrickGrid.load_npz(tmp_path / "bad.npz")


def test_hdf5_needs_h5py(tmp_path):
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(RuntimeError, match="h5py is required"):
            bn.torus_brick(3, 3, 3, spin_a=0.3).save_hdf5(tmp_path / "b.h5")
    else:
        pytest.skip("h5py present")


def test_tiles_and_levels():
    t = tiles.generate_tiles(130, 70, 64)
    assert len(t) == 3 * 2 and sum(x.pixels for x in t) == 130 * 70
    assert t[0] == tiles.RenderTile(0, 0, 0, 64, 64) and t[-1].x1 == 130 and t[-1].y1 == 70
    assert tiles.progressive_levels(1920, 1080, 480) == [(0, 480, 270), (1, 960, 540), (2, 1920, 1080)]
    assert tiles.progressive_levels(300, 200, 480) == [(0, 300, 200)]
    pt = list(tiles.generate_progressive_tiles(1024, 512, 256, 256))
    assert [x.level for x in pt] == [0] * 1 + [1] * 2 + [2] * 8
    views = tiles.tile_views(bn.View(130, 70), t)
    assert [v.rect for v in views][1] == (64, 0, 64, 64)


@pytest.mark.gpu
def test_progressive_render_levels_equal_plain_renders():
    b = bn.torus_brick(32, 16, 32, spin_a=0.9375, seed=4)
    db = bn.DeviceBrick(b)
    view = bn.View(256, 128, max_steps=2000)
    got = list(tiles.progressive_render(db, view, min_width=64))
    assert [lv for lv, _ in got] == [0, 1, 2]
    for (lv, img), (_, w, h) in zip(got, tiles.progressive_levels(256, 128, 64)):
        assert img.shape == (h, w, 4)
        from dataclasses import replace

        assert np.array_equal(img.cpu().numpy(), bn.render(db, replace(view, width=w, height=h)).image().cpu().numpy())
    # a tiled render of the full level equals the untiled image
    tv = tiles.tile_views(view, tiles.generate_tiles(256, 128, 64))
    res = bn.render(db, tv)
    full = bn.render(db, view).image().cpu().numpy()
    for i, t in enumerate(tiles.generate_tiles(256, 128, 64)):
        assert np.array_equal(res.image(i).cpu().numpy(), full[t.y0:t.y1, t.x0:t.x1])


@pytest.mark.gpu
def test_device_brick_from_reference_file():
    db = bn.DeviceBrick.from_npz(Path(__file__).parent / "golden" / "reference_brick.npz")
    assert db.shape == (4, 3, 5)
