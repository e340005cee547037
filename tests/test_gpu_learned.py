"""GPU checks of the learned step-size subsystem.

* training kernels: loss and gradient equal the float64 oracle's
  (oracle/mlp.py) to 1e-2 relative L2 (BF16 tanh of the kernels vs the
  oracle's correctly rounded tanh);
* inference (warp-level BF16 mma.sync): equals the oracle's forward to 3e-2;
* the step-doubling controller records finite samples and renders a finite
  image; training on them lowers the loss;
* the learned ray loop stays within tolerance of the FP64 plain method at a
  4x finer step.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import blackhole_native as bn
from blackhole_native import learned
from oracle import mlp as M
from tests.conftest import rel_l1
from tests.test_gpu_render import conditioned_pixels

pytestmark = pytest.mark.gpu


def _rand_net(seed=0):
    norm = np.zeros(18, dtype=np.float32)
    norm[8:16] = 1.0
    norm[17] = 1.0
    net = learned.StepNet.initial(norm, seed=seed)
    rng = np.random.default_rng(seed + 1)
    p = net.params.cpu().numpy()
    p[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, 64)
    p[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.1, 64)
    p[M.OFF_B3] = 0.3
    net.params.copy_(torch.from_numpy(p))
    return net


def test_grad_kernel_matches_oracle():
    L = learned._declare()
    net = _rand_net(3)
    rng = np.random.default_rng(7)
    n = 640
    rows = np.zeros((n, 9), dtype=np.float32)
    rows[:, :8] = rng.normal(size=(n, 8))
    rows[:, 8] = rng.normal(size=n)
    data = torch.from_numpy(rows).cuda()
    index = torch.arange(n, dtype=torch.int64, device="cuda")
    grad = torch.zeros(int(L.bhn_mlp_param_count()), dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    from blackhole_native import _device as dev, _lib

    _lib.check(L.bhn_mlp_grad(dev.ptr(net.params), dev.ptr(data), dev.ptr(index), 0, n, dev.ptr(grad),
                              dev.ptr(loss), dev.stream_ptr()))
    torch.cuda.synchronize()
    want_loss, want_grad = M.loss_and_grad(net.params.cpu().numpy(), rows[:, :8].astype(np.float64),
                                           rows[:, 8].astype(np.float64))
    got = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) / n - want_loss) <= 1e-2 * want_loss
    assert np.linalg.norm(got - want_grad) <= 1e-2 * np.linalg.norm(want_grad)
    for lo, hi in ((M.OFF_W1, M.OFF_B1), (M.OFF_W2, M.OFF_B2), (M.OFF_W3, M.OFF_B3)):
        cos = np.dot(got[lo:hi], want_grad[lo:hi]) / (np.linalg.norm(got[lo:hi]) * np.linalg.norm(want_grad[lo:hi]))
        assert cos > 0.999


def test_inference_matches_oracle():
    net = _rand_net(5)
    rng = np.random.default_rng(11)
    x = rng.normal(size=(1000, 8)).astype(np.float32)
    got = net.infer(torch.from_numpy(x)).cpu().numpy()
    want, _ = M.forward(net.params.cpu().numpy(), x.astype(np.float64))
    assert np.max(np.abs(got - want)) <= 3e-2 * max(1.0, np.max(np.abs(want)))
    assert np.mean(np.abs(got - want)) <= 5e-3 * max(1.0, np.mean(np.abs(want)))


@pytest.fixture(scope="module")
def scene3():
    brick = bn.torus_brick(128, 64, 128, spin_a=0.998, seed=1)
    return bn.DeviceBrick(brick, precisions=("fp32", "fp64"))


def test_controller_samples_and_training(scene3):
    view = bn.View(96, 96, spin_a=0.998, inclination_deg=60.0, max_steps=8192, horizon_guard=True)
    samples = learned.generate_samples(scene3, [view], learned.AdaptConfig(tol=1e-4, sample_prob=0.5), 200_000)
    assert samples.shape[0] > 20_000
    assert torch.isfinite(samples).all()
    # log(h_opt / h_plain) with h_opt in [h_floor, h_ceil] = [1e-6, 64], h_plain in [h_min, h_max] = [1e-3, 1]
    logm = samples[:, 8]
    assert float(logm.min()) >= np.log(1e-6) - 1e-3 and float(logm.max()) <= np.log(64.0 / 1e-3) + 1e-3
    net = learned.train(samples, epochs=4, batch=2048, lr=3e-3)
    assert net.losses[-1] < 0.5 * net.losses[0] and net.losses[-1] < 0.25
    run = learned.render_adaptive(scene3, [view], learned.AdaptConfig(tol=1e-4))
    assert torch.isfinite(run.image()).all()
    assert run.counters["steps"] > 0


def test_learned_loop_within_tolerance(scene3):
    view = bn.View(96, 96, spin_a=0.998, inclination_deg=60.0, max_steps=8192, horizon_guard=True)
    samples = learned.generate_samples(scene3, [view], learned.AdaptConfig(tol=1e-4, sample_prob=0.5), 200_000)
    net = learned.train(samples, epochs=4, batch=2048, lr=3e-3)
    run = learned.render_learned(scene3, [view], net, learned.AdaptConfig(tol=1e-4, margin=0.5, interval=2,
                                                                          check_tol=1e-2))
    img = run.image().cpu().numpy().astype(np.float64)
    ref = bn.render(scene3, view.scaled_step(0.25), precision="fp64").image().cpu().numpy()
    assert np.all(np.isfinite(img))
    cond = conditioned_pixels(scene3, view.scaled_step(0.25), ref)
    assert cond.mean() >= 0.98
    assert rel_l1(img[..., 0][cond], ref[..., 0][cond]) <= 2e-2
    assert run.counters["steps"] > 0 and run.counters["net_evals_per_warp"] > 0
