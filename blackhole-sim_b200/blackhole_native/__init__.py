"""blackhole_native -- B200 (sm_100a) drop-in for the reference's native core.

Importing this module is what python/blackhole_sim/native_loader.py:13-17
does (``importlib.import_module("blackhole_native")``); the functions below
are the ones native_kernels.py then calls, with the same arguments, errors
and output layout, computed by hand-written CUDA kernels.  There is no CPU
fallback: without the CUDA library the import fails, without a GPU every
compute call raises RuntimeError.

Exports beyond the reference's five:
  sample_brick_valid_mask  -- GPU form of native_kernels.py:189-210
  render / render_stokes / Renderer / DeviceBrick / View -- the fused
      persistent ray kernel over one or many views
"""

from __future__ import annotations

import platform as _platform
import sys as _sys

from . import _lib
from .bricks import COEFF_NAMES, BrickGrid, estimate_brick_memory, horizon_radius, torus_brick
from .kernels import (sample_and_step_stokes, sample_brick_trilinear, sample_brick_valid_mask, stokes_exact_brick,
                      stokes_rk2_brick)
from .render import (DeviceBrick, PipelinedRenderer, RenderConfig, Renderer, RenderResult, RenderStats, View, render,
                     render_stokes)
from . import accelerated, grrt, tiles
from .synchrotron import (HybridSynchrotronCoefficients, LocalPlasmaFrame, NonthermalPowerLawSynchrotronCoefficients,
                          PolarizedCoefficients, ThermalSynchrotronCoefficients, precompute_coefficient_bricks,
                          precompute_device_brick)

_lib.lib()  # fail loudly at import when the CUDA library is missing

__all__ = [
    "core_version", "detect_arch", "stokes_rk2_brick", "stokes_exact_brick", "sample_brick_trilinear", "sample_and_step_stokes",
    "sample_brick_valid_mask", "COEFF_NAMES", "BrickGrid", "estimate_brick_memory", "torus_brick", "horizon_radius",
    "DeviceBrick",
    "RenderConfig", "Renderer", "RenderResult", "RenderStats", "View", "render", "render_stokes", "PipelinedRenderer",
    "precompute_coefficient_bricks", "precompute_device_brick", "HybridSynchrotronCoefficients",
    "ThermalSynchrotronCoefficients", "NonthermalPowerLawSynchrotronCoefficients", "LocalPlasmaFrame",
    "PolarizedCoefficients", "accelerated", "grrt", "tiles",
]


def core_version() -> str:
    """Library version (native/core/src/lib.rs:19-22)."""
    return _lib.lib().bhn_core_version().decode()


def _normalized_arch(value: str) -> str:  # lib.rs:9-17
    return {"x86_64": "x86_64", "amd64": "x86_64", "aarch64": "arm64", "arm64": "arm64", "x86": "x86",
            "i386": "x86", "i686": "x86", "arm": "arm"}.get(value.lower(), "unknown")


def detect_arch() -> dict:
    """Host architecture of the loaded module (native/core/src/lib.rs:24-35)."""
    return {
        "arch": _normalized_arch(_platform.machine()),
        "os": _sys.platform if _sys.platform != "linux" else "linux",
        "family": "unix" if _sys.platform != "win32" else "windows",
        "pointer_width": str(64 if _sys.maxsize > 2 ** 32 else 32),
    }
