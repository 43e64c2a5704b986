"""The learned preconditioner on the device against its CPU restatement
(oracle/unet/unet_ref.py), and inside the solver.

* The tensor-core 3x3 convolution (tcgen05, BF16 operands, FP32 accumulator
  in TMEM) on host arrays: every output within one BF16 rounding of the
  float64 convolution of the same BF16 inputs (the device accumulates in FP32
  in another order, so a value next to a rounding boundary may round the other
  way), over shapes that take every path of the kernel -- partial tiles, one
  to nine taps per weight group, N from 16 to 128.
* The whole network's output and the gradient of its loss w.r.t. every
  weight, against the restatement with the device's BF16 roundings: output
  within 2e-2 relative L2, each layer's gradient within 5e-2 relative L2
  (cosine above 0.995) -- the BF16 activations between the layers are where
  the two part.
* Training on the device lowers the loss and the held-out error against the
  V-cycle; the trained network preconditions a flexible BiCGStab that meets the
  solve's tolerance, in fewer iterations than the method without it (the
  same Krylov iteration with the untrained network, and with diagonal
  scaling), and falls back to SA-AMG when capped.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

import _systems
import yuzen_b200 as yz
from yuzen_b200 import learned as yl

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "unet"))
import unet_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def _conv_ref(x, w, b, real_w, real_h, relu):
    H, W, cin = x.shape
    net = unet_ref.Net.__new__(unet_ref.Net)
    net.lv = [(H, W, real_h, real_w)]
    net.bf16 = True
    y = net.conv(unet_ref.to_bf16(x).reshape(H * W, cin), unet_ref.to_bf16(w),
                 None if b is None else b.astype(np.float32).astype(np.float64), 0, relu)
    return y.reshape(H, W, -1)


@pytest.mark.parametrize("H,W,cin,n,rw,rh,relu,bias", [
    (16, 24, 16, 16, 23, 16, True, True),
    (9, 40, 32, 64, 37, 8, True, True),      # partial last tile
    (8, 24, 128, 64, 20, 7, False, True),    # two weight groups (6 + 3 taps)
    (12, 20, 64, 128, 19, 12, False, False), # N = 128
    (10, 30, 48, 16, 29, 10, True, False),
    (6, 24, 96, 32, 22, 5, True, True),
    (3, 7, 16, 48, 6, 3, False, True),       # fewer pixels than a tile
])
def test_conv3x3_tensor_cores(H, W, cin, n, rw, rh, relu, bias):
    rng = np.random.default_rng(H * 1000 + cin + n)
    x = rng.standard_normal((H, W, cin)).astype(np.float32)
    x[rh:, :, :] = 0.0
    x[:, rw:, :] = 0.0
    w = (rng.standard_normal((n, 9, cin)) / np.sqrt(9 * cin)).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32) * 0.1 if bias else None
    y = yl.conv3x3(x, w, b, rw, rh, relu)
    ref = _conv_ref(x, w, b, rw, rh, relu)
    err = np.abs(y - ref)
    tol = np.abs(ref) * 2.0 ** -7 * 1.01 + 1e-6 * np.abs(ref).max()
    assert np.all(err <= tol), (err.max(), np.unravel_index(np.argmax(err - tol), err.shape))
    assert np.all(y[rh:, :, :] == 0) and np.all(y[:, rw:, :] == 0)


def _net_and_inputs(nx, ny, seed):
    rng = np.random.default_rng(seed)
    net = yl.UNet(nx, ny, capacity=4, seed=seed)
    p = unet_ref.init_params(seed).astype(np.float32)
    net.set_params(p)
    r = rng.standard_normal(nx * ny)
    # smooth-ish diagonal and height maps, as a film gives them
    diag = 1.0 + 1e3 * (1.0 + np.sin(np.arange(nx * ny) * 0.05)) ** 2
    h = 0.01 + np.abs(np.cos(np.arange(nx * ny) * 0.01))
    f, _ = yl.features(r, diag, h)
    return net, p.astype(np.float64), f, rng


@pytest.mark.parametrize("nx,ny", [(20, 18), (36, 36)])
def test_forward_matches_oracle(nx, ny):
    net, p, f, _ = _net_and_inputs(nx, ny, 7)
    out = net.forward(f)
    ref, _ = unet_ref.Net(nx, ny, bf16=True).forward(p, f.astype(np.float64))
    rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert rel < 2e-2, rel


@pytest.mark.parametrize("nx,ny", [(20, 18), (36, 36)])
def test_gradient_matches_oracle(nx, ny):
    net, p, f, rng = _net_and_inputs(nx, ny, 11)
    t = rng.standard_normal(nx * ny)
    loss, g = net.loss_grad(f, t)
    rl, rg = unet_ref.Net(nx, ny, bf16=True).loss_grad(p, f.astype(np.float64), t.astype(np.float32))
    assert abs(loss - rl) <= 1e-2 * abs(rl), (loss, rl)
    lay, ow, ob = unet_ref.param_layout()
    spans = [(a, b + unet_ref.CONVS[k][1]) for k, (a, b) in enumerate(lay)] + [(ow, ob + 1)]
    for a, b in spans:
        x, y = g[a:b].astype(np.float64), rg[a:b]
        rel = np.linalg.norm(x - y) / np.linalg.norm(y)
        cos = float(x @ y / (np.linalg.norm(x) * np.linalg.norm(y)))
        assert rel < 5e-2 and cos > 0.995, (a, b, rel, cos)


def _films(N, seeds, stiff=3.0):
    return [_systems.film_system(N, seed=s, stiff=stiff) for s in seeds]


def _pattern(d):
    return yz.CrsPattern(d["rowptr"], d["col"], d["sorted_col"], d["sorted_src"])


def test_training_lowers_the_loss():
    """Pairs (r, z) with z the film system's answer to r (solved to 1e-8),
    ten films; 300 Adam steps lower the loss and the held-out error."""
    N = 32
    nx = N + 4
    net = yl.UNet(nx, nx, capacity=32, seed=3)
    be = yz.B200Backend()
    rng = np.random.default_rng(0)
    for d in _films(N, range(10)):
        pat = _pattern(d)
        diag = d["values"][d["rowptr"][:-1]]
        for _ in range(3):
            r = rng.standard_normal(d["n"]) * (d["bc"] == 0)
            z = np.zeros(d["n"])
            be.Solve(yz.LinearSolverSettings(2, True, 200, 1e-8, False), pat, d["values"], r, z)
            net.add_sample(r / diag, z, diag)
    assert net.samples() == 30
    l0, v0 = net.train(1, batch=4, lr=1e-3, holdout=6)
    l1, v1 = net.train(300, batch=4, lr=1e-3, holdout=6)
    assert l1 < 0.5 * l0, (l0, l1)
    assert v1 < v0, (v0, v1)


def _solve(backend, d, rhs, s):
    x = np.zeros(d["n"])
    ret, it, res = backend.Solve(s, _pattern(d), d["values"], rhs, x)
    return ret, it, res, x


def test_learned_preconditioner_in_the_solver():
    """The network trained on the (residual, V-cycle) pairs the solver
    collects from its own SA-AMG solves of twelve films, then the
    preconditioner of a flexible BiCGStab on three held-out films: every solve
    meets the tolerance (its answer the AMG solve's to the tolerance's reach)
    in fewer iterations than the method without the trained network -- the
    same iteration with the untrained network, and BiCGStab with diagonal
    scaling -- and a cap it cannot meet hands the solve back to SA-AMG."""
    N = 44
    nx = N + 4
    s = yz.LinearSolverSettings(2, True, 3000, 1e-10, False)
    rng = np.random.default_rng(1)
    net = yl.UNet(nx, nx, capacity=96, seed=5)
    collect = yz.B200Backend()
    train_films = _films(N, range(12), stiff=2.0)
    collect.SetLearned(net, 1, collect_solves=len(train_films), per_solve=8)
    for d in train_films:
        ret, _, _, _ = _solve(collect, d, rng.standard_normal(d["n"]) * 1e-3 * (d["bc"] == 0), s)
        assert ret == 0
    assert net.samples() >= 40
    # the untrained network: the same seed, marked trained after no step
    untrained = yl.UNet(nx, nx, capacity=4, seed=5)
    d0 = train_films[0]
    for _ in range(3):
        untrained.add_sample(rng.standard_normal(d0["n"]), rng.standard_normal(d0["n"]), np.ones(d0["n"]))
    untrained.train(0, batch=1, lr=1e-3, holdout=1)
    loss, val = net.train(400, batch=4, lr=1e-3, holdout=8)
    assert 0 <= val < 1.0, val

    amg, learned_be, naive, jacobi = (yz.B200Backend() for _ in range(4))
    learned_be.SetLearned(net, 2, cap_factor=1e6)
    naive.SetLearned(untrained, 2, cap_factor=1e6)
    sj = yz.LinearSolverSettings(1, True, 3000, 1e-10, False)
    for d in _films(N, range(100, 103), stiff=2.0):
        rhs = rng.standard_normal(d["n"]) * 1e-3 * (d["bc"] == 0)
        ra, ia, _, xa = _solve(amg, d, rhs, s)
        rl, il, resl, xl = _solve(learned_be, d, rhs, s)
        rn, inn, _, _ = _solve(naive, d, rhs, s)
        rj, ij, _, _ = _solve(jacobi, d, rhs, sj)
        assert ra == 0 and rl == 0 and resl <= s.epsilon
        assert np.linalg.norm(xl - xa) <= 1e-6 * np.linalg.norm(xa)
        naive_its = inn if naive.learned_stats()["fallbacks"] == 0 else s.maxIteration
        jac_its = ij if rj == 0 else sj.maxIteration
        assert il < naive_its and il < jac_its, (il, naive_its, jac_its, ia)
    assert learned_be.learned_stats()["fallbacks"] == 0 and learned_be.learned_stats()["solves"] == 3
    # a cap the network cannot meet (one iteration): the solve goes back to SA-AMG
    learned_be.SetLearned(net, 2, cap_factor=1e-9)
    d = train_films[1]
    rhs = rng.standard_normal(d["n"]) * 1e-3 * (d["bc"] == 0)
    r, it, res, x = _solve(learned_be, d, rhs, s)
    assert r == 0 and res <= s.epsilon
    assert learned_be.learned_stats()["fallbacks"] == 1
