"""ctypes wrapper of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is a float64 C restatement of the
reference hot loop (see ``bhoracle.c`` for the per-function citations).  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker or the timed CPU
baseline -- never as the product path.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_lib = None

POLICY_CODES = {"nan": 0, "initial": 1, "zero": 2}
STATUS_NAMES = {0: "max_steps", 1: "captured", 2: "escaped", 3: "invalid", 4: "optically_thick"}


class View(ctypes.Structure):
    """Mirror of ``bho_view`` (bhoracle.h)."""

    _fields_ = [
        ("spin_a", ctypes.c_double),
        ("r_obs", ctypes.c_double),
        ("theta_obs", ctypes.c_double),
        ("phi_obs", ctypes.c_double),
        ("fov_y_deg", ctypes.c_double),
        ("roll_deg", ctypes.c_double),
        ("h_scale", ctypes.c_double),
        ("h_min", ctypes.c_double),
        ("h_max", ctypes.c_double),
        ("escape_radius", ctypes.c_double),
        ("affine_to_length_cm", ctypes.c_double),
        ("max_optical_depth", ctypes.c_double),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("x0", ctypes.c_int32),
        ("y0", ctypes.c_int32),
        ("crop_w", ctypes.c_int32),
        ("crop_h", ctypes.c_int32),
        ("max_steps", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


def build() -> Path:
    """Compile ``liboracle.so`` with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        d, i64, vp = ctypes.c_double, ctypes.c_int64, ctypes.c_void_p
        _lib.bho_render.argtypes = [ctypes.POINTER(View), vp, vp, i64, vp, i64, vp, i64, ctypes.c_int,
                                    ctypes.c_int, vp, vp, vp, vp]
        _lib.bho_render.restype = None
        _lib.bho_sample_brick_trilinear.argtypes = [vp, vp, i64, vp, i64, vp, i64, vp, i64, vp]
        _lib.bho_stokes_rk2_brick.argtypes = [vp, i64, d, vp, i64, vp]
        _lib.bho_sample_and_step_stokes.argtypes = [vp, vp, i64, vp, i64, vp, i64, vp, i64, d, vp, i64,
                                                    ctypes.c_int, vp]
        _lib.bho_sample_brick_valid_mask.argtypes = [vp, i64, vp, i64, vp, i64, vp]
        _lib.bho_geodesic_rhs.argtypes = [vp, d, d, d, vp]
        _lib.bho_rk2_step.argtypes = [vp, d, d, d, d, vp]
        _lib.bho_rk4_step.argtypes = [vp, d, d, d, d, vp]
        _lib.bho_trace_rk4.argtypes = [vp, d, d, d, d, ctypes.c_int32, d, vp, ctypes.POINTER(ctypes.c_int32)]
        _lib.bho_trace_rk4.restype = i64
        _lib.bho_hamiltonian.argtypes = [vp, d, d, d]
        _lib.bho_hamiltonian.restype = d
        _lib.bho_camera_ray.argtypes = [ctypes.POINTER(View), d, d, d, vp, ctypes.POINTER(d), ctypes.POINTER(d)]
        _lib.bho_camera_ray.restype = ctypes.c_int
        _lib.bho_metric_con.argtypes = [d, d, d, vp]
        _lib.bho_metric_cov.argtypes = [d, d, d, vp]
        _lib.bho_search_right.argtypes = [vp, i64, d]
        _lib.bho_search_right.restype = i64
        _lib.bho_max_threads.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def sample_brick_trilinear(coeffs, r_grid, theta_grid, phi_grid, points) -> np.ndarray:
    c, rg, tg, pg = _f64(coeffs), _f64(r_grid), _f64(theta_grid), _f64(phi_grid)
    pts = _f64(points).reshape(-1, 3)
    out = np.empty((pts.shape[0], 11), dtype=np.float64)
    lib().bho_sample_brick_trilinear(_p(c), _p(rg), rg.size, _p(tg), tg.size, _p(pg), pg.size, _p(pts),
                                     pts.shape[0], _p(out))
    return out


def stokes_rk2_brick(coeffs, ds_cm: float, initial) -> np.ndarray:
    c = _f64(coeffs).reshape(-1, 11)
    ini = _f64(initial).reshape(-1)
    out = np.empty((c.shape[0], 4), dtype=np.float64)
    lib().bho_stokes_rk2_brick(_p(c), c.shape[0], float(ds_cm), _p(ini), ini.size, _p(out))
    return out


def sample_and_step_stokes(coeffs, r_grid, theta_grid, phi_grid, points, ds_cm, initial, policy="nan"):
    c, rg, tg, pg = _f64(coeffs), _f64(r_grid), _f64(theta_grid), _f64(phi_grid)
    pts = _f64(points).reshape(-1, 3)
    ini = _f64(initial).reshape(-1)
    out = np.empty((pts.shape[0], 4), dtype=np.float64)
    lib().bho_sample_and_step_stokes(_p(c), _p(rg), rg.size, _p(tg), tg.size, _p(pg), pg.size, _p(pts),
                                     pts.shape[0], float(ds_cm), _p(ini), ini.size, POLICY_CODES[policy], _p(out))
    return out


def sample_brick_valid_mask(r_grid, theta_grid, points) -> np.ndarray:
    rg, tg = _f64(r_grid), _f64(theta_grid)
    pts = _f64(points).reshape(-1, 3)
    out = np.empty(pts.shape[0], dtype=np.uint8)
    lib().bho_sample_brick_valid_mask(_p(rg), rg.size, _p(tg), tg.size, _p(pts), pts.shape[0], _p(out))
    return out.astype(bool)


def geodesic_rhs(y, a, pt, pphi) -> np.ndarray:
    yy = _f64(y)
    out = np.empty(6)
    lib().bho_geodesic_rhs(_p(yy), a, pt, pphi, _p(out))
    return out


def rk2_step(y, h, a, pt, pphi) -> np.ndarray:
    yy = _f64(y)
    out = np.empty(6)
    lib().bho_rk2_step(_p(yy), h, a, pt, pphi, _p(out))
    return out


def trace_rk4(y0, pt, pphi, a, h, max_steps, escape_radius):
    """kerr.py:337-384 (store_stride 1): (states (n, 6), status 0..3)."""
    states = np.empty((int(max_steps) + 1, 6))
    st = ctypes.c_int32()
    n = lib().bho_trace_rk4(_p(_f64(y0)), pt, pphi, a, h, int(max_steps), escape_radius, _p(states), ctypes.byref(st))
    return states[:n].copy(), int(st.value)


def camera_ray(view, ndc_x, ndc_y, aspect):
    """kerr.py:188-233: (y0 (6,), p_t, p_phi)."""
    y0 = np.zeros(6)
    pt, pphi = ctypes.c_double(), ctypes.c_double()
    rc = lib().bho_camera_ray(ctypes.byref(view), ndc_x, ndc_y, aspect, _p(y0), ctypes.byref(pt), ctypes.byref(pphi))
    if rc != 0:
        raise ValueError("invalid camera")
    return y0, pt.value, pphi.value


def hamiltonian(y, a, pt, pphi) -> float:
    yy = _f64(y)
    return float(lib().bho_hamiltonian(_p(yy), a, pt, pphi))


def metric_con(r, th, a) -> np.ndarray:
    out = np.empty(16)
    lib().bho_metric_con(r, th, a, _p(out))
    return out.reshape(4, 4)


def metric_cov(r, th, a) -> np.ndarray:
    out = np.empty(16)
    lib().bho_metric_cov(r, th, a, _p(out))
    return out.reshape(4, 4)


def make_view(**kw) -> View:
    v = View()
    for k, val in kw.items():
        setattr(v, k, val)
    return v


def camera_ray(view: View, ndc_x: float, ndc_y: float, aspect: float):
    y0 = np.empty(6)
    pt, pphi = ctypes.c_double(), ctypes.c_double()
    rc = lib().bho_camera_ray(ctypes.byref(view), ndc_x, ndc_y, aspect, _p(y0), ctypes.byref(pt), ctypes.byref(pphi))
    if rc != 0:
        raise ValueError("camera tetrad undefined")
    return y0, pt.value, pphi.value


def render(view: View, coeffs, r_grid, theta_grid, phi_grid, *, stop_at_tau: bool = True, threads: int = 0):
    """Render ``view``'s crop rectangle.  Returns (stokes[h,w,4], steps[h,w], status[h,w], h_drift[h,w])."""
    c, rg, tg, pg = _f64(coeffs), _f64(r_grid), _f64(theta_grid), _f64(phi_grid)
    h, w = int(view.crop_h), int(view.crop_w)
    out = np.zeros((h, w, 4))
    steps = np.zeros((h, w), dtype=np.int32)
    status = np.zeros((h, w), dtype=np.int32)
    drift = np.zeros((h, w))
    lib().bho_render(ctypes.byref(view), _p(c), _p(rg), rg.size, _p(tg), tg.size, _p(pg), pg.size,
                     int(bool(stop_at_tau)), int(threads), _p(out), _p(steps), _p(status), _p(drift))
    return out, steps, status, drift


def max_threads() -> int:
    return int(lib().bho_max_threads())


def cpu_count() -> int:
    return len(os.sched_getaffinity(0))
