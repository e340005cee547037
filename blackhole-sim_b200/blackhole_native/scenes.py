"""Seeded synthetic scenes for the benchmark workloads.

* ``single_view_scene``: one 1024 x 1024 camera at r_obs = 1000 M, inclination
  17 deg, field of view +-20 M, a = 0.9375, RK2 h = 0.02 r in [1e-3, 1], 4096
  steps, through a 256 x 128 x 256 torus brick.
* ``uneven_views``: many views of uneven size, spin, inclination and step
  budget drawn from a seed, all through one shared brick.
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np

from .bricks import BrickGrid, torus_brick
from .render import FOV_20M_AT_1000M, View

SINGLE_VIEW = dict(width=1024, height=1024, spin_a=0.9375, r_obs=1000.0, inclination_deg=17.0, max_steps=4096,
                   h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0)


def single_view_scene(side: int = 1024, seed: int = 0) -> tuple[BrickGrid, View]:
    brick = torus_brick(256, 128, 256, spin_a=SINGLE_VIEW["spin_a"], seed=seed, dtype=np.float32)
    return brick, View(**{**SINGLE_VIEW, "width": side, "height": side})


def uneven_views(n: int = 256, seed: int = 0, side_range=(64, 1024), spin_range=(0.0, 0.998),
                 incl_range_deg=(5.0, 85.0), steps_range=(512, 8192)) -> list[View]:
    """n views with square side ~ U{64..1024}, spin ~ U(0, 0.998), inclination
    ~ U(5, 85) deg and max_steps ~ U{512..8192}, from numpy.random.default_rng(seed);
    every view uses the single-view camera distance, field of view and step law."""
    rng = np.random.default_rng(int(seed))
    sides = rng.integers(side_range[0], side_range[1] + 1, size=n)
    spins = rng.uniform(*spin_range, size=n)
    incl = rng.uniform(*incl_range_deg, size=n)
    steps = rng.integers(steps_range[0], steps_range[1] + 1, size=n)
    base = View(**SINGLE_VIEW)
    return [replace(base, width=int(s), height=int(s), spin_a=float(a), inclination_deg=float(i), max_steps=int(m))
            for s, a, i, m in zip(sides, spins, incl, steps)]


def shared_brick(nr: int = 128, ntheta: int = 64, nphi: int = 128, seed: int = 0) -> BrickGrid:
    """The brick every uneven view shares; its r grid starts at 1.05 r_+ of the
    largest spin drawn (a = 0.998), so it covers every view's exterior."""
    return torus_brick(nr, ntheta, nphi, spin_a=0.998, seed=seed, dtype=np.float32)


def total_pixels(views) -> int:
    return int(sum(v.pixels for v in views))


__all__ = ["single_view_scene", "uneven_views", "shared_brick", "total_pixels", "FOV_20M_AT_1000M"]
