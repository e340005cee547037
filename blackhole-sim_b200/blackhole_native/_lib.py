"""ctypes binding of ``libbhnative.so`` (include/blackhole_native.h).

Loading the library needs no GPU; every compute call does.  A missing library
is an ImportError and a missing GPU a RuntimeError: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libbhnative.so"

BHN_OK, BHN_ERR_VALUE, BHN_ERR_CUDA, BHN_ERR_DEVICE, BHN_ERR_UNSUPPORTED = range(5)
POLICY_CODES = {"nan": 0, "initial": 1, "zero": 2}
RAY_STATUS = ("max_steps", "captured", "escaped", "invalid", "optically_thick")

# Every symbol include/blackhole_native.h declares.
EXPORTED = (
    "bhn_core_version", "bhn_last_error", "bhn_device_info", "bhn_fp32_peak_probe", "bhn_fp64_peak_probe",
    "bhn_stokes_rk2_brick", "bhn_stokes_exact_brick", "bhn_sample_brick_trilinear", "bhn_sample_and_step_stokes",
    "bhn_sample_sort_scratch_bytes", "bhn_sample_and_step_stokes_sorted", "bhn_sample_brick_trilinear_sorted",
    "bhn_sample_brick_valid_mask", "bhn_check_values",
    "bhn_brick_tables_bytes", "bhn_brick_build_tables", "bhn_brick_pack", "bhn_brick_locate",
    "bhn_render_scratch_bytes", "bhn_render_prepare", "bhn_render_launch", "bhn_render_noalloc",
    "bhn_graph_create", "bhn_graph_launch", "bhn_graph_destroy",
    "bhn_mlp_param_count", "bhn_mlp_blob_bytes", "bhn_mlp_pack", "bhn_mlp_grad", "bhn_mlp_adam", "bhn_mlp_infer",
    "bhn_adaptive_launch", "bhn_learned_launch", "bhn_brick_precompute", "bhn_synchrotron_coefficients",
    "bhn_grrt_scratch_bytes", "bhn_grrt_render", "bhn_brick_trace_render",
)
NOALLOC_MAX_VIEWS = 120  # BHN_NOALLOC_MAX_VIEWS


class ViewStruct(ctypes.Structure):
    """``bhn_view``."""

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
        ("out_offset", ctypes.c_int64),
    ]


class RenderConfigStruct(ctypes.Structure):
    """``bhn_render_config``."""

    _fields_ = [
        ("block_threads", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("tile_w", ctypes.c_int32),
        ("tile_h", ctypes.c_int32),
        ("refill_min", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("reg_cap", ctypes.c_int32),
    ]


class RenderStatsStruct(ctypes.Structure):
    """``bhn_render_stats`` (read back from the device)."""

    _fields_ = [
        ("ray_steps", ctypes.c_ulonglong),
        ("brick_steps", ctypes.c_ulonglong),
        ("rays", ctypes.c_ulonglong),
        ("status", ctypes.c_ulonglong * 5),
        ("queue_fetches", ctypes.c_ulonglong),
        ("max_h_drift", ctypes.c_float),
        ("error_flags", ctypes.c_uint32),
        ("max_h_drift_escaped", ctypes.c_float),
        ("pad0", ctypes.c_uint32),
    ]


class RayOutputsStruct(ctypes.Structure):
    """``bhn_ray_outputs``."""

    _fields_ = [
        ("steps", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("h_drift", ctypes.c_void_p),
    ]


STATS_BYTES = ctypes.sizeof(RenderStatsStruct)

_lib: ctypes.CDLL | None = None


def _declare(lib: ctypes.CDLL) -> None:
    vp, i64, i32, d = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
    sig = {
        "bhn_core_version": ([], ctypes.c_char_p),
        "bhn_last_error": ([], ctypes.c_char_p),
        "bhn_device_info": ([vp, vp, vp, vp], ctypes.c_int),
        "bhn_fp32_peak_probe": ([vp, i32, i32, vp, vp], ctypes.c_int),
        "bhn_fp64_peak_probe": ([vp, i32, i32, i32, vp, vp], ctypes.c_int),
        "bhn_stokes_rk2_brick": ([vp, i64, d, vp, i64, vp, vp], ctypes.c_int),
        "bhn_stokes_exact_brick": ([vp, i64, d, vp, i64, vp, vp], ctypes.c_int),
        "bhn_sample_brick_trilinear": ([vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp], ctypes.c_int),
        "bhn_sample_and_step_stokes": ([vp, vp, i64, vp, i64, vp, i64, vp, i64, d, vp, i64, i32, vp, vp],
                                       ctypes.c_int),
        "bhn_sample_sort_scratch_bytes": ([i64, i64], ctypes.c_int64),
        "bhn_sample_brick_trilinear_sorted": ([vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp, i64, vp], ctypes.c_int),
        "bhn_sample_and_step_stokes_sorted": ([vp, vp, i64, vp, i64, vp, i64, vp, i64, d, vp, i64, i32, vp, vp, i64,
                                               vp], ctypes.c_int),
        "bhn_sample_brick_valid_mask": ([vp, i64, vp, i64, vp, i64, vp, vp], ctypes.c_int),
        "bhn_check_values": ([vp, i64, i32, vp, vp], ctypes.c_int),
        "bhn_brick_tables_bytes": ([i32, i32, i32], i64),
        "bhn_brick_build_tables": ([vp, i32, vp, i32, vp, i32, vp, vp], ctypes.c_int),
        "bhn_brick_pack": ([vp, i32, i64, vp, i32, vp, vp], ctypes.c_int),
        "bhn_brick_locate": ([vp, i32, i32, i32, vp, i64, vp, vp, vp], ctypes.c_int),
        "bhn_render_scratch_bytes": ([i32], i64),
        "bhn_render_prepare": ([ctypes.POINTER(ViewStruct), i32, vp, i64, vp], ctypes.c_int),
        "bhn_render_launch": ([vp, vp, i32, i32, i32, i32, ctypes.POINTER(RenderConfigStruct), vp,
                               ctypes.POINTER(RayOutputsStruct), vp, i64, vp, vp], ctypes.c_int),
        "bhn_render_noalloc": ([vp, vp, i32, i32, i32, ctypes.POINTER(ViewStruct), i32,
                                ctypes.POINTER(RenderConfigStruct), vp, ctypes.POINTER(RayOutputsStruct), vp, vp],
                               ctypes.c_int),
        "bhn_graph_create": ([vp, vp, i32, i32, i32, i32, ctypes.POINTER(RenderConfigStruct), vp,
                              ctypes.POINTER(RayOutputsStruct), vp, i64, vp, ctypes.POINTER(vp)], ctypes.c_int),
        "bhn_graph_launch": ([vp, vp], ctypes.c_int),
        "bhn_graph_destroy": ([vp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        try:
            fn = getattr(lib, name)
        except AttributeError as exc:
            raise ImportError(f"blackhole_native: {LIB_PATH} lacks {name}; the library is older than its "
                              "binding -- rebuild it with `python blackhole-sim_b200/blackhole_native/_build.py`") from exc
        fn.argtypes = args
        fn.restype = res


def lib() -> ctypes.CDLL:
    """Load (once) and return the CUDA library."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"blackhole_native: CUDA library {LIB_PATH} is missing; build it with "
                "`python blackhole-sim_b200/blackhole_native/_build.py` (nvcc, sm_100a)")
        handle = ctypes.CDLL(str(LIB_PATH))
        _declare(handle)
        _lib = handle
    return _lib


def last_error() -> str:
    raw = lib().bhn_last_error()
    return raw.decode("utf-8", "replace") if raw else ""


def check(rc: int) -> None:
    """Raise the Python exception matching a bhn_status."""
    if rc == BHN_OK:
        return
    msg = last_error()
    if rc == BHN_ERR_VALUE:
        raise ValueError(msg)
    raise RuntimeError(f"blackhole_native: {msg} (status {rc})")
