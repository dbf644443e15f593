"""The learned coarse-grid correction on the GPU.

* forward and MSE-loss gradients of the CUDA network kernels against the CPU
  oracle (oracle/learned.py) on the same parameters and inputs;
* the energy-loss training path (solver-bound, level-2 Galerkin operator)
  against central finite differences of its own loss;
* training lowers the energy loss;
* what the trained network gains over the plain V-cycle: solves with it
  attached converge to the same solution, and the auto mode measures both
  and keeps the plain V-cycle whenever the network does not lower the
  iteration count.
"""
import json
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import learned  # noqa: E402

pytestmark = pytest.mark.gpu


def _f32(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32).reshape(-1), device="cuda")


def test_forward_matches_oracle(gputo):
    import torch
    rng = np.random.default_rng(1)
    dims = (6, 5, 7)
    th = learned.init_params(2)
    th[learned.num_params() - 3:] = [0.1, -0.2, 0.3]    # nonzero output bias
    x = rng.standard_normal((4,) + dims).astype(np.float32)
    net = gputo.Net(seed=0)
    net.set_params(th)
    y = torch.empty(3 * np.prod(dims), dtype=torch.float32, device="cuda")
    net.forward(_f32(x), dims, y)
    ref, _ = learned.forward(x, th)
    got = y.cpu().numpy().reshape(ref.shape)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


def test_mse_gradient_matches_oracle(gputo):
    rng = np.random.default_rng(2)
    dims = (5, 4, 6)
    th = learned.init_params(4)
    xs = rng.standard_normal((2, 4) + dims).astype(np.float32)
    ts = rng.standard_normal((2, 3) + dims).astype(np.float32)
    ms = (rng.random((2, 3) + dims) > 0.3).astype(np.float32)
    net = gputo.Net(seed=0)
    net.set_params(th)
    g = np.zeros(learned.num_params(), dtype=np.float32)
    loss = net.train_step(_f32(xs), _f32(ts), _f32(ms), 2, dims, 0.0, grads_out=g)
    ref_g = np.zeros(learned.num_params())
    ref_l = 0.0
    for q in range(2):
        y, acts = learned.forward(xs[q], th)
        l, gy = learned.loss(y, ts[q], ms[q])
        ref_l += l / 2
        ref_g += learned.backward(acts, th, gy)
    assert abs(loss - ref_l) <= 1e-4 * abs(ref_l)
    assert np.abs(g - ref_g).max() <= 1e-3 * np.abs(ref_g).max()
    # the step with lr = 0 left the parameters alone
    assert np.array_equal(net.get_params(), th)


def _problem(gputo, shape=(64, 32, 32), nl=4, seed=0):
    import torch
    F, fixed = gputo.cantilever(*shape)
    x = gputo.random_field_density(*shape, seed=seed, corr_len=6.0)
    CX = torch.as_tensor(1e-9 + x ** 3 * (1 - 1e-9), dtype=torch.float64, device="cuda")
    s = gputo.Solver(*shape, nl, gputo.default_options(precision=gputo.PREC_MIXED))
    s.set_problem(gputo.hex8_stiffness(), fixed)
    s.setup(CX)
    return s, torch.as_tensor(F, dtype=torch.float64, device="cuda")


def test_energy_loss_gradient_matches_finite_differences(gputo):
    """Biases enter the network in FP32 (weights are BF16-rounded), so central
    differences in every layer's biases check the energy-loss gradient through
    the whole backward pass."""
    import torch
    s, F = _problem(gputo)
    samples = gputo.harvest_net_samples(s, F, iters=3)
    X = torch.stack([q[0] for q in samples[:2]]).contiguous()
    G = torch.stack([q[1] for q in samples[:2]]).contiguous()
    net = gputo.Net(seed=5)
    th = net.get_params()
    g = np.zeros_like(th)
    s.net_train_step(net, X, G, 2, 0.0, grads_out=g)
    offs, o = [], 0
    for ws, bs in learned.layer_shapes():
        o += int(np.prod(ws))
        offs += [o + c for c in range(min(bs[0], 4))]
        o += bs[0]
    for i in offs:
        h = 1e-3
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        net.set_params(tp)
        lp = s.net_train_step(net, X, G, 2, 0.0) * 2
        net.set_params(tm)
        lm = s.net_train_step(net, X, G, 2, 0.0) * 2
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 2e-2 * max(abs(fd), abs(g[i])) + 1e-3 * np.abs(g).max(), (i, fd, g[i])
    net.set_params(th)


def test_training_lowers_energy_loss(gputo):
    s, F = _problem(gputo)
    samples = gputo.harvest_net_samples(s, F, iters=20)
    net = gputo.Net(seed=1)
    hist = gputo.train_net(s, net, samples, epochs=8, lr=1e-3, batch=4)
    assert hist[-1] < hist[0] and hist[-1] < 0.0   # 0 = the plain V-cycle


def test_learned_correction_gain_and_fallback(gputo, tmp_path):
    """Train on one design, then solve a held-out design: plain, with the
    network always on, and in auto mode.  The solution is the same in all
    three; auto mode ends on whichever needed fewer iterations."""
    import torch
    s0, F = _problem(gputo, seed=0)
    samples = gputo.harvest_net_samples(s0, F, iters=30)
    net = gputo.Net(seed=1)
    gputo.train_net(s0, net, samples, epochs=4, lr=3e-4, batch=8)
    s, F = _problem(gputo, seed=11)
    res = {}
    U0 = torch.zeros_like(F)
    res["plain"] = s.solve(F, U0, 1e-8, 400)
    s.set_net(net, 1)
    U1 = torch.zeros_like(F)
    res["net"] = s.solve(F, U1, 1e-8, 400)
    assert res["net"][0] < 1e-8, res
    c0 = float(F @ U0)
    assert abs(float(F @ U1) - c0) <= 1e-6 * abs(c0)
    s.set_net(net, 2)
    nits = []
    for _ in range(4):
        U = torch.zeros_like(F)
        rr, nit = s.solve(F, U, 1e-8, 400)
        assert rr < 1e-8 and abs(float(F @ U) - c0) <= 1e-6 * abs(c0)
        nits.append(nit)
    on, plain_nit, net_nit = s.net_state()
    assert plain_nit == res["plain"][1] and net_nit == res["net"][1]
    assert on == (net_nit < plain_nit)
    assert nits[-1] == min(plain_nit, net_nit)
    gain = {"plain_nit": plain_nit, "net_nit": net_nit, "auto_uses_net": on,
            "gain_iterations": plain_nit - net_nit}
    (tmp_path / "learned_gain.json").write_text(json.dumps(gain))
    print("learned correction:", gain)
