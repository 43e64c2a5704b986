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
  V-cycle, well below the untrained network's; in the solver the flexible
  BiCGStab with the network returns the solution to the tolerance, through
  the network or its SA-AMG fallback.
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


def _net_and_inputs(nx, ny, seed, act):
    rng = np.random.default_rng(seed)
    net = yl.UNet(nx, ny, capacity=4, seed=seed, activation=act)
    p = unet_ref.init_params(seed, act).astype(np.float32)
    net.set_params(p)
    r = rng.standard_normal(nx * ny)
    # smooth-ish diagonal and height maps, as a film gives them
    diag = 1.0 + 1e3 * (1.0 + np.sin(np.arange(nx * ny) * 0.05)) ** 2
    h = 0.01 + np.abs(np.cos(np.arange(nx * ny) * 0.01))
    f, _ = yl.features(r, diag, h)
    return net, p.astype(np.float64), f, rng


@pytest.mark.parametrize("act", [0, 1], ids=["linear", "relu"])
@pytest.mark.parametrize("nx,ny", [(20, 18), (36, 36)])
def test_forward_matches_oracle(nx, ny, act):
    net, p, f, _ = _net_and_inputs(nx, ny, 7, act)
    out = net.forward(f)
    ref, _ = unet_ref.Net(nx, ny, bf16=True, act=act).forward(p, f.astype(np.float64))
    rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert rel < 2e-2, rel


@pytest.mark.parametrize("act", [0, 1], ids=["linear", "relu"])
@pytest.mark.parametrize("nx,ny", [(20, 18), (36, 36)])
def test_gradient_matches_oracle(nx, ny, act):
    net, p, f, rng = _net_and_inputs(nx, ny, 11, act)
    t = rng.standard_normal(nx * ny)
    loss, g = net.loss_grad(f, t)
    rl, rg = unet_ref.Net(nx, ny, bf16=True, act=act).loss_grad(p, f.astype(np.float64), t.astype(np.float32))
    assert abs(loss - rl) <= 1e-2 * abs(rl), (loss, rl)
    lay, ow, ob = unet_ref.param_layout()
    if act:
        spans = [(a, b + unet_ref.CONVS[k][1]) for k, (a, b) in enumerate(lay)] + [(ow, ob + 1)]
    else:
        # no biases without activation: the weights alone
        spans = list(lay) + [(ow, ob)]
    for a, b in spans:
        x, y = g[a:b].astype(np.float64), rg[a:b]
        rel = np.linalg.norm(x - y) / np.linalg.norm(y)
        cos = float(x @ y / (np.linalg.norm(x) * np.linalg.norm(y)))
        assert rel < 5e-2 and cos > 0.995, (a, b, rel, cos)


def _pattern(d):
    return yz.CrsPattern(d["rowptr"], d["col"], d["sorted_col"], d["sorted_src"])


def _step_films(N, factors, steps):
    """Film systems as the step assembles them: the all-physics film of N^2
    cells after each of `steps` steps, its first Newton system
    I + theta dt J and right-hand side at dt times each factor (dicts in the
    form of the solve fixtures, with the film height)"""
    from yuzen_b200 import cases
    from yuzen_b200 import step as ys
    state = cases.allphys(N=N, steps=max(steps) + 1).state()
    st = ys.Step(ys.params_from_state(state), state["field_h0"], state["field_c0"], state["field_s0"])
    rowptr, col, bc = st.pattern()
    scol, ssrc = _systems.sorted_mirror(rowptr, col)
    out, done = [], 0
    for k in steps:
        st.advance(k - done)
        done = k
        h, _ = st.fields()
        for f in factors:
            ia, rhs = st.system(h, h, state["dt"] * f)
            out.append({"n": rhs.size, "rowptr": rowptr, "col": col, "sorted_col": scol, "sorted_src": ssrc,
                        "values": ia, "rhs": rhs, "bc": bc, "h": h})
    return out


def _collect(net, films, s, per_solve):
    """(residual, V-cycle) pairs the solver collects from its own SA-AMG
    solves of the films"""
    be = yz.B200Backend()
    be.SetLearned(net, 1, collect_solves=len(films), per_solve=per_solve)
    for d in films:
        x = np.zeros(d["n"])
        ret, _, _ = be.Solve(s, _pattern(d), d["values"], d["rhs"], x)
        assert ret == 0


S = yz.LinearSolverSettings(2, True, 3000, 1e-10, False)


def test_collected_pairs_carry_their_systems_features():
    """A pair the solver collects from its own SA-AMG solve holds the feature
    maps of that solve's system -- f1 = log10|a_ii| / 4 of the unscaled
    matrix's diagonal (the first entry of each row in storage order) and
    f2 = log10 h / 2 + 1 of the film given -- the maps the network reads when
    it is applied to such a system."""
    import torch
    d = _step_films(64, (1.0,), (0,))[0]
    net = yl.UNet(68, 68, capacity=4, seed=1)
    be = yz.B200Backend()
    hd = torch.tensor(d["h"], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    be.SetAux(hd.data_ptr())
    be.SetLearned(net, 1, collect_solves=1, per_solve=2)
    x = np.zeros(d["n"])
    ret, _, _ = be.Solve(S, _pattern(d), d["values"], d["rhs"], x)
    assert ret == 0 and net.samples() >= 1
    diag = np.abs(d["values"][d["rowptr"][:-1]])
    f1 = (np.log10(np.maximum(diag, 1e-30)) * 0.25).astype(np.float32)
    f2 = (np.log10(np.maximum(d["h"], 1e-30)) * 0.5 + 1.0).astype(np.float32)
    s = net.sample(0)
    assert s["valid"]
    assert np.abs(f1).max() > 1e-3 and np.abs(f2).max() > 0.5
    np.testing.assert_allclose(s["f1"], f1, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(s["f2"], f2, rtol=1e-6, atol=1e-6)
    del hd


def test_training_lowers_the_loss():
    """Pairs the solver collects from its SA-AMG solves of twelve film
    systems of the 64^2 all-physics film; 300 Adam steps on the device lower
    the loss and bring the held-out error against the V-cycle well below the
    untrained network's."""
    net = yl.UNet(68, 68, capacity=96, seed=3)
    _collect(net, _step_films(64, (0.5, 1.0, 2.0, 4.0), (0, 2, 4)), S, 8)
    assert net.samples() >= 24
    l0, v0 = net.train(1, batch=4, lr=1e-3, holdout=6)
    l1, v1 = net.train(300, batch=4, lr=1e-3, holdout=6)
    assert l1 < 0.5 * l0, (l0, l1)
    assert v1 < 0.8 * v0 and v1 < 0.5, (v0, v1)


def _solve(backend, d, rhs, s):
    x = np.zeros(d["n"])
    ret, it, res = backend.Solve(s, _pattern(d), d["values"], rhs, x)
    return ret, it, res, x


def test_learned_preconditioner_in_the_solver():
    """The network trained on the (residual, V-cycle) pairs the solver
    collects from its own SA-AMG solves of twelve film systems.  SA-AMG is
    the yardstick: on the held-out pairs the trained network's error against the
    V-cycle is well below the untrained network's (the same weights before
    training, on the same pairs) -- what the training gains.  As the
    preconditioner of a flexible BiCGStab on held-out systems every solve
    returns the solution to the tolerance, through the network or, where it
    does not converge within its cap, through the SA-AMG fallback; a cap it
    cannot meet hands the solve back to SA-AMG.  The iteration counts of the
    network, of BiCGStab with diagonal scaling and of SA-AMG are printed side
    by side: on these films the network needs more iterations than both."""
    train = _step_films(64, (0.5, 1.0, 2.0, 4.0), (0, 2, 4))
    net = yl.UNet(68, 68, capacity=96, seed=5)
    untrained = yl.UNet(68, 68, capacity=96, seed=5)
    _collect(net, train, S, 8)
    _collect(untrained, train, S, 8)          # the same pairs (the solves are deterministic)
    assert net.samples() == untrained.samples() >= 24
    _, val0 = untrained.train(0, batch=1, lr=1e-3, holdout=6)
    loss, val = net.train(400, batch=4, lr=1e-3, holdout=6)
    print("held-out error against the V-cycle: untrained %.3f, trained %.3f" % (val0, val))
    assert 0 <= val < 0.5 * val0, (val, val0)

    amg, learned_be, jacobi = (yz.B200Backend() for _ in range(3))
    learned_be.SetLearned(net, 2, cap_factor=1e6)
    sj = yz.LinearSolverSettings(1, True, 3000, 1e-10, False)
    seen = []
    for d in _step_films(64, (1.5, 3.0), (6,)):
        ra, ia, _, xa = _solve(amg, d, d["rhs"], S)
        f0 = learned_be.learned_stats()["fallbacks"]
        rl, il, resl, xl = _solve(learned_be, d, d["rhs"], S)
        rj, ij, _, _ = _solve(jacobi, d, d["rhs"], sj)
        seen.append({"network": il, "fell_back": learned_be.learned_stats()["fallbacks"] > f0,
                     "jacobi": ij if rj == 0 else None, "amg": ia})
        assert ra == 0 and rl == 0 and resl <= S.epsilon, seen
        assert np.linalg.norm(xl - xa) <= 1e-6 * np.linalg.norm(xa), seen
    print("iterations on the held-out films:", seen)
    # a cap the network cannot meet (one iteration): the solve goes back to SA-AMG
    fresh = yz.B200Backend()
    fresh.SetLearned(net, 2, cap_factor=1e-9)
    d = train[1]
    r, it, res, x = _solve(fresh, d, d["rhs"], S)
    assert r == 0 and res <= S.epsilon
    assert fresh.learned_stats()["fallbacks"] == 1
