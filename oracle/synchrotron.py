"""CPU oracle of the coefficient-brick precompute (test infrastructure only).

float64 numpy restatement of the reference's brick precompute
(python/blackhole_sim/coefficient_bricks.py:110-152) with its Hybrid
synchrotron model (python/blackhole_sim/synchrotron.py:120-325).  Only tests
import this module; the product path is the CUDA kernel behind
``bhn_brick_precompute``.

Third-party arithmetic restated here:
* ``scipy.special.kv`` (scipy 1.18 in the reference's environment) for
  K_{2/3} in the G(x) = x K_{2/3}(x) kernel table: evaluated from the integral
  representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt (DLMF 10.32.9)
  by the trapezoid rule, which converges geometrically for this analytic,
  doubly-exponentially decaying integrand.
* ``scipy.special.kv(2, 1/Theta_e)`` normalises the thermal distribution
  (synchrotron.py:189-196), which is then normalised again by its own
  trapezoid integral; the first factor cancels exactly and is left out.
* ``numpy.polynomial.legendre.leggauss`` (Gauss-Legendre pitch nodes) and
  ``numpy.interp`` / ``numpy.trapezoid`` / ``numpy.geomspace`` are numpy's own
  and are called as the reference calls them.
"""

from __future__ import annotations

import math

import numpy as np

# python/blackhole_sim/calibration.py:18-25
C_CGS = 2.99792458e10
M_PROTON_CGS = 1.67262192369e-24
M_ELECTRON_CGS = 9.1093837015e-28
K_BOLTZMANN_CGS = 1.380649e-16
E_CHARGE_ESU = 4.80320471257e-10
H_PLANCK_CGS = 6.62607015e-27  # synchrotron.py:177

TABLE_N = 256  # synchrotron.py:158 (_synchrotron_kernel_table default)

THERMAL = dict(gamma_grid_size=192, pitch_nodes=16, faraday_rotation_scale=1.0, faraday_conversion_scale=1.0)
NONTHERMAL = dict(p=3.5, gamma_min=10.0, gamma_max=1.0e5, nonthermal_fraction=0.02, gamma_grid_size=224,
                  pitch_nodes=16, absorption_scale=1.0, faraday_scale=0.15)


def kv(nu: float, x: np.ndarray) -> np.ndarray:
    """K_nu(x) for x > 0 from DLMF 10.32.9 by the trapezoid rule.  The step is
    scaled with the integrand's width (~1/sqrt(x) near t = 0 for large x) and
    the range ends where x (cosh t - 1) passes 750."""
    x = np.asarray(x, dtype=float)
    out = np.empty_like(x)
    for i, xi in np.ndenumerate(x):
        h = min(0.02, 0.25 / math.sqrt(xi))
        t_max = math.acosh(1.0 + 750.0 / xi)
        t = np.arange(0.0, t_max + h, h)
        y = np.exp(-xi * np.cosh(t)) * np.cosh(nu * t)
        out[i] = h * (0.5 * y[0] + y[1:].sum())
    return out


def synchrotron_f(x):
    """synchrotron.py:120-136: 1.25 x^(1/3) exp(-x) (648 + x^2)^(1/12), x clipped to [1e-12, 1e3]."""
    xx = np.clip(np.asarray(x, dtype=float), 1.0e-12, 1.0e3)
    out = 1.25 * np.power(xx, 1.0 / 3.0) * np.exp(-xx) * np.power(648.0 + xx * xx, 1.0 / 12.0)
    return np.nan_to_num(out, nan=0.0, posinf=0.0, neginf=0.0)


def synchrotron_g(x):
    """synchrotron.py:139-155: G(x) = x K_{2/3}(x), x clipped to [1e-12, 1e3]."""
    xx = np.clip(np.asarray(x, dtype=float), 1.0e-12, 1.0e3)
    out = xx * kv(2.0 / 3.0, xx)
    return np.nan_to_num(out, nan=0.0, posinf=0.0, neginf=0.0)


def kernel_table(n: int = TABLE_N):
    """synchrotron.py:157-162."""
    xs = np.geomspace(1.0e-8, 1.0e3, n)
    return xs, synchrotron_f(xs), synchrotron_g(xs)


_TABLE = None


def kernel_interp(x):
    """synchrotron.py:165-172: log-log linear interpolation of the F/G table."""
    global _TABLE
    if _TABLE is None:
        _TABLE = kernel_table()
    xs, F, G = _TABLE
    lx = np.log(np.clip(np.asarray(x, dtype=float), xs[0], xs[-1]))
    lxs = np.log(xs)
    outF = np.exp(np.interp(lx, lxs, np.log(np.maximum(F, 1.0e-300))))
    outG = np.exp(np.interp(lx, lxs, np.log(np.maximum(G, 1.0e-300))))
    return outF, outG


def planck_nu(nu_hz: float, theta_e: float) -> float:
    """synchrotron.py:175-182."""
    T = theta_e * M_ELECTRON_CGS * C_CGS * C_CGS / K_BOLTZMANN_CGS
    x = H_PLANCK_CGS * nu_hz / max(K_BOLTZMANN_CGS * T, 1.0e-300)
    if x < 1.0e-3:
        return 2.0 * nu_hz * nu_hz * K_BOLTZMANN_CGS * T / (C_CGS * C_CGS)
    return 2.0 * H_PLANCK_CGS * nu_hz ** 3 / (C_CGS * C_CGS) / max(math.expm1(min(x, 700.0)), 1.0e-300)


def integrated_j(n_e, b_gauss, nu_hz, gamma, f_gamma, pitch_nodes):
    """synchrotron.py:185-237: pitch-averaged j_I and j_Q (cos_pitch_to_los = 0)."""
    if n_e <= 0.0 or b_gauss <= 0.0:
        return 0.0, 0.0
    mu, w = np.polynomial.legendre.leggauss(pitch_nodes)
    total_I = total_Q = 0.0
    nu_B = E_CHARGE_ESU * b_gauss / (2.0 * math.pi * M_ELECTRON_CGS * C_CGS)
    for m, ww in zip(mu, w):
        sin_a = math.sqrt(max(0.0, 1.0 - float(m) ** 2))
        Bp = b_gauss * sin_a
        if Bp <= 0.0:
            continue
        nu_c = 1.5 * gamma * gamma * nu_B * sin_a
        x = nu_hz / np.maximum(nu_c, 1.0e-300)
        F, G = kernel_interp(x)
        pref = math.sqrt(3.0) * E_CHARGE_ESU ** 3 * Bp / (M_ELECTRON_CGS * C_CGS ** 2)
        total_I += 0.5 * ww * float(np.trapezoid(f_gamma * pref * F, gamma))
        total_Q += 0.5 * ww * float(np.trapezoid(f_gamma * pref * G, gamma))
    return n_e * total_I / (4.0 * math.pi), n_e * total_Q / (4.0 * math.pi)


def _rotated(c, chi):
    """synchrotron.py:67-77 (PolarizedCoefficients.rotated)."""
    co, si = math.cos(2.0 * chi), math.sin(2.0 * chi)
    ji, jq, ju, jv, ai, aq, au, av, rv, rq, ru = c
    return np.array([ji, jq * co - ju * si, jq * si + ju * co, jv, ai, aq * co - au * si, aq * si + au * co, av,
                     rv, rq * co - ru * si, rq * si + ru * co])


def thermal(n_e, theta_e, b_gauss, evpa, nu_hz, m=THERMAL, cos_los=0.0):
    """synchrotron.py:189-196, 248-275 (brick frames have cos_pitch_to_los = 0)."""
    if n_e <= 0.0 or b_gauss <= 0.0 or nu_hz <= 0.0:
        return np.zeros(11)
    gmax = max(10.0, 1.0 + 45.0 * theta_e)
    gamma = 1.0 + np.geomspace(1.0e-5, gmax - 1.0, m["gamma_grid_size"])
    beta = np.sqrt(np.maximum(1.0 - 1.0 / np.maximum(gamma, 1.0) ** 2, 0.0))
    f = gamma * gamma * beta * np.exp(-gamma / max(theta_e, 1.0e-12))
    integ = np.trapezoid(f, gamma)
    f = f / integ if integ > 0.0 else f
    jI, jQ0 = integrated_j(n_e, b_gauss, nu_hz, gamma, f, m["pitch_nodes"])
    Bnu = planck_nu(nu_hz, theta_e)
    alphaI = jI / max(Bnu, 1.0e-300)
    alphaQ0 = jQ0 / max(Bnu, 1.0e-300)
    b_perp = abs(b_gauss) * math.sqrt(max(0.0, 1.0 - cos_los ** 2))  # synchrotron.py:37-43
    b_par = b_gauss * cos_los
    rel_supp = max(1.0 / (theta_e * theta_e + 1.0), 1.0e-8)
    rhoV = m["faraday_rotation_scale"] * (E_CHARGE_ESU ** 3 / (math.pi * M_ELECTRON_CGS ** 2 * C_CGS ** 2))
    rhoV *= n_e * b_par / max(nu_hz * nu_hz, 1.0e-300) * rel_supp
    rhoQ = m["faraday_conversion_scale"] * (E_CHARGE_ESU ** 4 / (4.0 * math.pi ** 2 * M_ELECTRON_CGS ** 3 * C_CGS ** 3))
    rhoQ *= n_e * b_perp ** 2 / max(nu_hz ** 3, 1.0e-300) * max(theta_e, 1.0e-8)
    c = [max(jI, 0.0), max(jQ0, 0.0), 0.0, 0.0, max(alphaI, 0.0), max(alphaQ0, 0.0), 0.0, 0.0, rhoV, rhoQ, 0.0]
    return _rotated(c, evpa)


def nonthermal(n_e, theta_e, b_gauss, evpa, nu_hz, m=NONTHERMAL, cos_los=0.0):
    """synchrotron.py:199-204, 290-311."""
    if n_e <= 0.0 or b_gauss <= 0.0 or nu_hz <= 0.0 or m["nonthermal_fraction"] <= 0.0:
        return np.zeros(11)
    p, gmin, gmax = m["p"], m["gamma_min"], m["gamma_max"]
    gamma = np.geomspace(gmin, gmax, m["gamma_grid_size"])
    mask = (gamma >= gmin) & (gamma <= gmax)
    f = np.zeros_like(gamma)
    f[mask] = gamma[mask] ** (-p)
    f = f / max(np.trapezoid(f, gamma), 1.0e-300)
    n_s = n_e * m["nonthermal_fraction"]
    jI, jQ0 = integrated_j(n_s, b_gauss, nu_hz, gamma, f, m["pitch_nodes"])
    b_perp = abs(b_gauss) * math.sqrt(max(0.0, 1.0 - cos_los ** 2))
    b_par = b_gauss * cos_los
    char_gamma = max(gmin, math.sqrt(max(nu_hz / max(4.2e6 * b_perp, 1.0e-300), 1.0)))
    energy = char_gamma * M_ELECTRON_CGS * C_CGS * C_CGS
    alphaI = m["absorption_scale"] * jI / max(energy * nu_hz * nu_hz / (C_CGS * C_CGS), 1.0e-300)
    pol_frac = min((p + 1.0) / (p + 7.0 / 3.0), 0.85)
    jQ0 = min(jQ0, pol_frac * jI)
    alphaQ0 = min(alphaI * pol_frac, alphaI)
    rhoV = m["faraday_scale"] * (E_CHARGE_ESU ** 3 / (math.pi * M_ELECTRON_CGS ** 2 * C_CGS ** 2))
    rhoV *= n_s * b_par / max(nu_hz * nu_hz, 1.0e-300) / max(gmin ** 2, 1.0)
    rhoQ = m["faraday_scale"] * (E_CHARGE_ESU ** 4 / (4.0 * math.pi ** 2 * M_ELECTRON_CGS ** 3 * C_CGS ** 3))
    rhoQ *= n_s * b_perp ** 2 / max(nu_hz ** 3, 1.0e-300) * math.log(max(gmax / gmin, 1.0))
    c = [max(jI, 0.0), max(jQ0, 0.0), 0.0, 0.0, max(alphaI, 0.0), max(alphaQ0, 0.0), 0.0, 0.0, rhoV, rhoQ, 0.0]
    return _rotated(c, evpa)


def cell_frame(rho, theta_e, b_con, rho_cgs_per_code, b_gauss_per_code, mu_e=1.0):
    """coefficient_bricks.py:110-116 (_fast_frame) with calibration.py:113-119."""
    b_vec = np.asarray(b_con[1:], dtype=float)
    b_code = float(np.linalg.norm(b_vec))
    b_gauss = b_code * b_gauss_per_code
    n_e = rho * rho_cgs_per_code / max(mu_e * M_PROTON_CGS, 1.0e-300)
    evpa = float(np.arctan2(b_vec[2], b_vec[1])) if b_code > 0.0 else 0.0
    return n_e, max(theta_e, 1.0e-8), max(b_gauss, 0.0), evpa


def precompute(rho, theta_e, b_con, nu_hz, rho_cgs_per_code, b_gauss_per_code, mu_e=1.0, dtype="float32",
               stride=1):
    """coefficient_bricks.py:119-152 with the Hybrid model: (nr, nt, np, 11)."""
    sl = (slice(None, None, stride),) * 3
    rho, theta_e, b_con = rho[sl], theta_e[sl], b_con[sl]
    out_dtype = np.dtype(dtype)
    out = np.zeros(rho.shape + (11,), dtype=out_dtype)
    for idx in np.ndindex(rho.shape):
        n_e, te, b, evpa = cell_frame(float(rho[idx]), float(theta_e[idx]), b_con[idx], rho_cgs_per_code,
                                      b_gauss_per_code, mu_e)
        out[idx] = thermal(n_e, te, b, evpa, nu_hz) + nonthermal(n_e, te, b, evpa, nu_hz)
    big = np.finfo(out_dtype).max
    return np.nan_to_num(out, nan=0.0, posinf=big, neginf=0.0)
