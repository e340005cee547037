"""Shared test helpers: views of the golden fixtures and oracle adapters."""

from __future__ import annotations

import math

import numpy as np

from oracle import oracle as O


def golden_view(g, name: str):
    """(package View kwargs, oracle View) for a ray-loop fixture."""
    W, H, r_obs, inc, fov, a, ms, hs, hmin, hmax, esc, x0, y0, cw, ch = g[f"{name}_view"]
    kw = dict(width=int(W), height=int(H), r_obs=float(r_obs), inclination_deg=float(inc), fov_y_deg=float(fov),
              spin_a=float(a), max_steps=int(ms), h_scale=float(hs), h_min=float(hmin), h_max=float(hmax),
              escape_radius=float(esc), crop=(int(x0), int(y0), int(cw), int(ch)))
    return kw, oracle_view(**kw)


def oracle_view(*, width, height, r_obs=1000.0, inclination_deg=17.0, phi_deg=0.0, fov_y_deg=None, roll_deg=0.0,
                spin_a=0.9375, max_steps=4096, h_scale=0.02, h_min=1e-3, h_max=1.0, escape_radius=220.0,
                affine_to_length_cm=1.0, max_optical_depth=30.0, crop=None, horizon_guard=False):
    if fov_y_deg is None:
        fov_y_deg = 2.0 * math.degrees(math.atan(20.0 / 1000.0))
    x0, y0, cw, ch = crop if crop is not None else (0, 0, width, height)
    return O.make_view(spin_a=spin_a, r_obs=r_obs, theta_obs=math.radians(inclination_deg),
                       phi_obs=math.radians(phi_deg), fov_y_deg=fov_y_deg, roll_deg=roll_deg, h_scale=h_scale,
                       h_min=h_min, h_max=h_max, escape_radius=escape_radius,
                       affine_to_length_cm=affine_to_length_cm, max_optical_depth=max_optical_depth, width=width,
                       height=height, x0=x0, y0=y0, crop_w=cw, crop_h=ch, max_steps=max_steps,
                       flags=1 if horizon_guard else 0)


def view_to_oracle(v):
    """Oracle view for a blackhole_native.View."""
    return oracle_view(width=v.width, height=v.height, r_obs=v.r_obs, inclination_deg=v.inclination_deg,
                       phi_deg=v.phi_deg, fov_y_deg=v.fov_y_deg, roll_deg=v.roll_deg, spin_a=v.spin_a,
                       max_steps=v.max_steps, h_scale=v.h_scale, h_min=v.h_min, h_max=v.h_max,
                       escape_radius=v.escape_radius, affine_to_length_cm=v.affine_to_length_cm,
                       max_optical_depth=v.max_optical_depth, crop=v.rect, horizon_guard=v.horizon_guard)


def linear_coeff_fixture(nphi: int = 2):
    """The reference's sampler test fixture (python/tests/test_native_sampler_parity.py:22-35)."""
    r_grid = np.array([0.0, 1.0])
    theta_grid = np.array([0.0, 1.0])
    phi_grid = np.array([0.0, 1.0]) if nphi == 2 else np.linspace(0.0, 2.0 * math.pi, nphi, endpoint=False)
    coeffs = np.empty((2, 2, nphi, 11))
    for ir in range(2):
        for it in range(2):
            for ip in range(nphi):
                coeffs[ir, it, ip] = 100.0 * ir + 10.0 * it + ip + np.arange(11) * 0.125
    return coeffs, r_grid, theta_grid, phi_grid


def rust_linear_fixture():
    """The Rust core's unit-test fixture (native/core/src/lib.rs:384-397)."""
    c = []
    for ir in range(2):
        for it in range(2):
            for ip in range(2):
                base = ir * 100.0 + it * 10.0 + ip
                c.extend(base + k * 0.001 for k in range(11))
    return np.array(c)


def pol_fraction(img):
    """Linear polarization fraction m = sqrt(Q^2 + U^2) / I (polarized_transfer.py:41-44)."""
    I = np.maximum(img[..., 0], 1e-300)
    return np.sqrt(img[..., 1] ** 2 + img[..., 2] ** 2) / I


def flux_weighted_dm(a, b, floor: float = 1e-6):
    """Flux-weighted mean |m_a - m_b| (weights I_b) over the pixels that carry
    flux: I_b and I_a above ``floor`` times the peak I_b (the polarization
    fraction of a pixel with no intensity is undefined)."""
    Ib = b[..., 0]
    if not np.any(Ib > 0):
        return 0.0
    lit = (Ib > floor * Ib.max()) & (a[..., 0] > floor * Ib.max())
    w = np.where(lit, Ib, 0.0)
    if w.sum() <= 0:
        return 0.0
    dm = np.abs(pol_fraction(a) - pol_fraction(b))
    return float(np.sum(w[lit] * dm[lit]) / np.sum(w[lit]))
