"""The allocation-free render entry point (bhn_render_noalloc).

Callers that cannot allocate device memory -- a host whose device memory
belongs to its own allocator or to a pool sized at start-up, or a real-time
loop that may not take the synchronisation an allocation can imply -- pass
only inputs and outputs; the scratch lives in a fixed array inside the
library.  These tests call it through the C ABI twice in a row and compare
each result with the regular entry point's (bhn_render_prepare +
bhn_render_launch with caller-allocated scratch): the kernel, launch shape
and inputs are the same, so the images are bit-identical.  They also check
that a call changes neither torch's allocation count nor the device's free
memory, and that the largest view count the fixed array allows renders.  The
file sits apart, collected last, and passes alone or after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import blackhole_native as bn
from blackhole_native import _lib

pytestmark = pytest.mark.gpu


def _views():
    return [bn.View(96, 64, max_steps=2000, crop=(16, 8, 64, 48)),
            bn.View(40, 32, r_obs=60.0, fov_y_deg=30.0, inclination_deg=70.0, spin_a=0.5, max_steps=900)]


def _structs(views):
    offsets, total = [], 0
    for v in views:
        offsets.append(total)
        total += v.pixels
    return (_lib.ViewStruct * len(views))(*[v.to_struct(o) for v, o in zip(views, offsets)]), total


def _noalloc(db, arr, n, cstruct, out, stats):
    rc = _lib.lib().bhn_render_noalloc(db.records("fp32").data_ptr(), db.tables.data_ptr(), db.nr, db.nt, db.np, arr,
                                       n, ctypes.byref(cstruct), out.data_ptr(), None,
                                       stats.data_ptr() if stats is not None else None,
                                       torch.cuda.current_stream().cuda_stream)
    _lib.check(rc)


def test_noalloc_render_matches_allocating_entry_point():
    brick = bn.torus_brick(64, 32, 64, spin_a=0.9375, seed=3)
    db = bn.DeviceBrick(brick, precisions=("fp32",))
    views = _views()
    cfg = bn.RenderConfig()
    reference = bn.render(db, views, precision="fp32", config=cfg)
    want = reference.out.clone()
    torch.cuda.synchronize()
    assert float(want[:, 0].abs().sum()) > 0.0

    arr, total = _structs(views)
    cstruct = cfg.to_struct(0)
    outs = [torch.full((total, 4), float("nan"), dtype=torch.float32, device="cuda") for _ in range(2)]
    stats = [torch.zeros(_lib.STATS_BYTES, dtype=torch.uint8, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for k in range(2):  # two calls in a row share the library's scratch array
        allocated = torch.cuda.memory_allocated()
        free_before = torch.cuda.mem_get_info()[0]
        _noalloc(db, arr, len(views), cstruct, outs[k], stats[k])
        torch.cuda.synchronize()
        if k == 1:  # the first call on the device may still load the module; the second allocates nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        assert torch.cuda.memory_allocated() == allocated
        assert torch.equal(outs[k], want)
        st = bn.RenderStats.from_device(stats[k])
        assert st.rays == total and st.ray_steps == reference.stats().ray_steps


def test_noalloc_render_at_the_view_limit():
    brick = bn.torus_brick(16, 8, 16, spin_a=0.9375, seed=5)
    db = bn.DeviceBrick(brick, precisions=("fp32",))
    n = _lib.NOALLOC_MAX_VIEWS
    views = [bn.View(4 + i % 3, 3 + i % 2, r_obs=40.0 + i, inclination_deg=10.0 + 0.5 * i, fov_y_deg=40.0,
                     max_steps=300) for i in range(n)]
    cfg = bn.RenderConfig()
    want = bn.render(db, views, precision="fp32", config=cfg).out.clone()
    arr, total = _structs(views)
    cstruct = cfg.to_struct(0)
    for _ in range(2):
        out = torch.full((total, 4), float("nan"), dtype=torch.float32, device="cuda")
        _noalloc(db, arr, n, cstruct, out, None)
        torch.cuda.synchronize()
        assert torch.equal(out, want)


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
