"""The C-ABI library: it loads without a GPU, exports every symbol the public
header declares, and its struct layouts match the ctypes mirrors."""

from __future__ import annotations

import ctypes
import re
import shutil
import subprocess

import pytest

from tests.conftest import REPO

HEADER = REPO / "include" / "blackhole_native.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(bhn_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("bhn_stokes_rk2_brick", "bhn_sample_brick_trilinear", "bhn_sample_and_step_stokes",
                 "bhn_sample_brick_valid_mask", "bhn_render_launch", "bhn_core_version"):
        assert must in names


def test_library_loads_and_exports_every_declared_symbol():
    from blackhole_native import _lib

    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) == set(declared_functions())


def test_version_and_arch_without_gpu():
    import blackhole_native as bn

    assert bn.core_version().startswith("0.9.0")
    arch = bn.detect_arch()
    assert set(arch) == {"arch", "os", "family", "pointer_width"}


def test_sizes_without_gpu():
    from blackhole_native import _lib

    lib = _lib.lib()
    assert lib.bhn_render_scratch_bytes(0) == 0
    assert lib.bhn_render_scratch_bytes(1) > 0
    assert lib.bhn_render_scratch_bytes(256) > lib.bhn_render_scratch_bytes(1)
    nb = lib.bhn_brick_tables_bytes(256, 128, 256)
    assert nb % 16 == 0 and nb >= 128 + 12 * (256 + 128 + 256)
    from blackhole_native import grrt

    g = grrt._declare()
    one, four = g.bhn_grrt_scratch_bytes(14400, 1), g.bhn_grrt_scratch_bytes(14400, 4)
    assert 0 < one < four and four - one >= 3 * 14400 * grrt.SEGMENT_BYTES
    assert g.bhn_grrt_scratch_bytes(-1, 1) == -1 and g.bhn_grrt_scratch_bytes(10, 0) == -1
    assert grrt.default_chunk(14400) == 198 and grrt.default_chunk(10**7) == 16 and grrt.default_chunk(1) == 256


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_struct_layouts_match_ctypes(tmp_path):
    from blackhole_native import _lib

    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "blackhole_native.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(bhn_view), sizeof(bhn_render_config),"
        " sizeof(bhn_render_stats), sizeof(bhn_ray_outputs), offsetof(bhn_view, out_offset),"
        " offsetof(bhn_render_stats, max_h_drift)); return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(_lib.ViewStruct), ctypes.sizeof(_lib.RenderConfigStruct),
            ctypes.sizeof(_lib.RenderStatsStruct), ctypes.sizeof(_lib.RayOutputsStruct),
            _lib.ViewStruct.out_offset.offset, _lib.RenderStatsStruct.max_h_drift.offset]
    assert got == want


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_parameter_struct_layouts_match_ctypes(tmp_path):
    """bhn_adapt_params and bhn_synchrotron_model against their ctypes mirrors."""
    from blackhole_native import learned, synchrotron

    src = tmp_path / "sizes2.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "blackhole_native.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(bhn_adapt_params),"
        " offsetof(bhn_adapt_params, fallback), offsetof(bhn_adapt_params, seed), sizeof(bhn_synchrotron_model),"
        " offsetof(bhn_synchrotron_model, nonthermal_gamma_n), offsetof(bhn_synchrotron_model, nonthermal_faraday_scale));"
        " return 0;}\n")
    exe = tmp_path / "sizes2"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    A, M = learned.AdaptStruct, synchrotron.ModelStruct
    want = [ctypes.sizeof(A), A.fallback.offset, A.seed.offset, ctypes.sizeof(M), M.nonthermal_gamma_n.offset,
            M.nonthermal_faraday_scale.offset]
    assert got == want


def test_compute_calls_fail_loudly_without_gpu():
    import torch

    import blackhole_native as bn

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA GPU"):
        bn.stokes_rk2_brick([1.0] * 11, 0.1, [0.0] * 4)
    with pytest.raises(RuntimeError, match="CUDA GPU"):
        bn.sample_brick_valid_mask([0.0, 1.0], [0.0, 1.0], [0.5, 0.5, 0.5])
