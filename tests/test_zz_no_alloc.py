"""The allocation-free render entry point (bhn_render_noalloc).

Callers that cannot allocate device memory -- code that runs while a stream is
being captured into a CUDA graph, or a host whose device memory belongs to its
own allocator -- pass only inputs and outputs; the scratch lives in a fixed
array inside the library.  This test calls it through the C ABI twice in a row
and compares each result with the regular entry point's (bhn_render_prepare +
bhn_render_launch with caller-allocated scratch).  It sits in its own file,
collected last, and passes alone or after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import blackhole_native as bn
from blackhole_native import _lib
from tests.conftest import rel_l1

pytestmark = pytest.mark.gpu


def _views():
    return [bn.View(96, 64, max_steps=2000, crop=(16, 8, 64, 48)),
            bn.View(40, 32, r_obs=60.0, fov_y_deg=30.0, inclination_deg=70.0, spin_a=0.5, max_steps=900)]


def test_noalloc_render_matches_allocating_entry_point():
    brick = bn.torus_brick(64, 32, 64, spin_a=0.9375, seed=3)
    db = bn.DeviceBrick(brick, precisions=("fp32",))
    views = _views()
    cfg = bn.RenderConfig()
    reference = bn.render(db, views, precision="fp32", config=cfg)
    want = reference.out.clone()
    torch.cuda.synchronize()
    assert float(want[:, 0].abs().sum()) > 0.0

    offsets, total = [], 0
    for v in views:
        offsets.append(total)
        total += v.pixels
    arr = (_lib.ViewStruct * len(views))(*[v.to_struct(o) for v, o in zip(views, offsets)])
    cstruct = cfg.to_struct(0)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the library's scratch array
        out = torch.full((total, 4), float("nan"), dtype=torch.float32, device="cuda")
        stats = torch.zeros(_lib.STATS_BYTES, dtype=torch.uint8, device="cuda")
        rc = L.bhn_render_noalloc(db.records("fp32").data_ptr(), db.tables.data_ptr(), db.nr, db.nt, db.np, arr,
                                  len(views), ctypes.byref(cstruct), out.data_ptr(), None, stats.data_ptr(), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        assert np.all(np.isfinite(got))
        assert rel_l1(got, want.cpu().numpy()) <= 1e-6   # the FP32 kernel's own tolerance is 1e-3
        st = bn.RenderStats.from_device(stats)
        assert st.rays == total and st.ray_steps == reference.stats().ray_steps


def test_noalloc_render_rejects_too_many_views():
    brick = bn.torus_brick(8, 6, 8, spin_a=0.9375, seed=3)
    db = bn.DeviceBrick(brick, precisions=("fp32",))
    n = _lib.NOALLOC_MAX_VIEWS + 1
    v = bn.View(4, 4, max_steps=10)
    arr = (_lib.ViewStruct * n)(*[v.to_struct(16 * i) for i in range(n)])
    out = torch.zeros((16 * n, 4), dtype=torch.float32, device="cuda")
    cstruct = bn.RenderConfig().to_struct(0)
    rc = _lib.lib().bhn_render_noalloc(db.records("fp32").data_ptr(), db.tables.data_ptr(), db.nr, db.nt, db.np,
                                       arr, n, ctypes.byref(cstruct), out.data_ptr(), None, None,
                                       torch.cuda.current_stream().cuda_stream)
    with pytest.raises(ValueError, match="views per call"):
        _lib.check(rc)
