"""bench.py's host-side pieces that need no GPU: the CPU-baseline leg of the
brick-renderer workload (the oracle on a bounded sample) and its workload
constants."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

REPO = Path(__file__).resolve().parents[1]


def test_bricks_cpu_baseline_contract():
    sys.path.insert(0, str(REPO))
    import bench
    from blackhole_native import accelerated as acc
    from blackhole_native import bricks

    b = bricks.torus_brick(16, 8, 16, spin_a=0.9375, seed=0, dtype=np.float32)
    grid = SimpleNamespace(r=b.r, theta=b.theta, phi=b.phi, coeffs=b.coeffs)
    cfg = acc.AcceleratedRenderConfig(width=8, height=4, max_steps=300)
    out = bench.bricks_cpu_baseline(grid, SimpleNamespace(spin_a=0.9375), cfg, target_s=0.2)
    assert set(out) == {"value", "unit", "cores", "kind", "sample"}
    assert out["unit"] == "pixels/s" and out["cores"] == 1 and out["kind"] == "port" and out["value"] > 0
    assert "oracle/bricktrace.py" in out["sample"]


def test_bench_lists_the_bricks_workload():
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), "--help"], capture_output=True, text=True,
                         check=True).stdout
    assert "bricks" in out and "micro" in out and "--workload" in out
    import bench

    assert bench.FP64_FLOP_PER_RK4_STEP > 4 * 100 and bench.FP64_FLOP_PER_SEGMENT > 7 * 11 * 3
    json.dumps(bench.BRICKS_BRICK)


def test_micro_cpu_baseline_contract():
    sys.path.insert(0, str(REPO))
    import bench
    from blackhole_native import bricks

    b = bricks.torus_brick(8, 6, 8, spin_a=0.9375, seed=0, dtype=np.float64)
    rng = np.random.default_rng(1)
    pts = np.stack([rng.uniform(b.r[0], b.r[-1], 5000), rng.uniform(b.theta[0], b.theta[-1], 5000),
                    rng.uniform(0.0, 6.28, 5000)], axis=1)
    out = bench.micro_cpu_baseline(b, pts, 0.05, target_s=0.05)
    assert set(out) == {"value", "unit", "cores", "kind", "sample"}
    assert out["unit"] == "points/s" and out["cores"] == 1 and out["value"] > 0
    assert bench.MICRO_BYTES_PER_POINT == 3 * 8 + 8 * 11 * 8 + 4 * 8


def test_reference_arm_runs_without_the_cuda_library():
    """The reference arm times the oracle only: it must not import the package
    (which loads libbhnative.so).  Run on a small brick in a fresh process."""
    code = (
        "import sys, json, io, contextlib\n"
        f"sys.path.insert(0, {str(REPO)!r})\n"
        "import bench\n"
        "bench.BRICK.update(nr=16, ntheta=8, nphi=16)\n"
        "bench.WORKLOAD.update(max_steps=400)\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.main(['--impl', 'reference', '--steps', '1', '--warmup', '3', '--ref-seconds', '0.1'])\n"
        "line = json.loads(buf.getvalue().strip().splitlines()[-1])\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'impl': line['impl'], 'value': line['value'], 'pkg': 'blackhole_native' in sys.modules,\n"
        "                  'so': 'libbhnative' in maps, 'oracle': 'liboracle' in maps}))\n"
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True, cwd=str(REPO))
    got = json.loads(out.stdout.strip().splitlines()[-1])
    assert got["impl"] == "reference" and got["value"] > 0
    assert got["oracle"] and not got["pkg"] and not got["so"]
