"""The CPU restatement of the learned preconditioner's network
(oracle/unet/unet_ref.py) pinned on the CPU: its image geometry keeps a zero
column right of the real region at every level (so the device's linear-index
convolution is a zero-padded one), its BF16 rounding is round-to-nearest-even,
and its analytic gradient matches central finite differences of its own
float64 loss.  The device's gradients are held to this restatement
(tests/test_unet_gpu.py)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "unet"))
import unet_ref  # noqa: E402


@pytest.mark.parametrize("nx,ny", [(10, 10), (13, 9), (68, 68), (516, 516), (228, 228)])
def test_geometry(nx, ny):
    lv = unet_ref.geometry(nx, ny)
    assert lv[0][2:] == (ny, nx)
    for H, W, rh, rw in lv:
        assert W >= rw + 1 and H >= rh and W % 1 == 0
    for a, b in zip(lv, lv[1:]):
        assert (b[0] * 2, b[1] * 2) == (a[0], a[1])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159265, 1e-3], dtype=np.float64)
    r = unet_ref.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # a tie rounds to even
    assert r[2] == 1.0 + 2 ** -7                 # above the tie rounds up
    assert r[3] == -2.5
    assert abs(r[4] - np.pi) <= 2 ** -7 * 4
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


@pytest.mark.parametrize("act", [0, 1])
def test_gradient_matches_finite_differences(act):
    nx = ny = 10
    net = unet_ref.Net(nx, ny, bf16=False, act=act)
    rng = np.random.default_rng(3)
    p = unet_ref.init_params(5, act)
    feat = rng.standard_normal((3, nx * ny))
    t = rng.standard_normal(nx * ny)
    loss, g = net.loss_grad(p, feat, t)
    lay, ow, ob = unet_ref.param_layout()
    weights = np.concatenate([np.arange(a, b) for a, b in lay] + [np.arange(ow, ow + 16)])
    # without activation the biases are held at 0 (their gradient is not computed)
    pool = np.arange(p.size) if act else weights
    idx = rng.choice(pool, 60, replace=False)
    idx = np.concatenate([idx, [p.size - 2] + ([p.size - 1] if act else [])])      # the output layer too
    eps = 1e-6
    worst = 0.0
    for k in idx:
        q = p.copy(); q[k] += eps
        lp = net.loss_grad(q, feat, t)[0]
        q[k] -= 2 * eps
        lm = net.loss_grad(q, feat, t)[0]
        fd = (lp - lm) / (2 * eps)
        worst = max(worst, abs(fd - g[k]) / max(1e-6, abs(fd) + abs(g[k])))
    assert worst < 1e-4, worst


def test_linear_network_is_linear_in_r():
    """Without activation the network is a linear operator on r (the input
    channels are r times functions of the features)."""
    nx = ny = 12
    net = unet_ref.Net(nx, ny, bf16=False, act=0)
    rng = np.random.default_rng(4)
    p = unet_ref.init_params(2, 0)
    f = rng.standard_normal((3, nx * ny))
    r1, r2 = rng.standard_normal(nx * ny), rng.standard_normal(nx * ny)
    out = lambda r: net.forward(p, np.stack([r, f[1], f[2]]))[0]
    a, b = 0.7, -2.3
    lhs = out(a * r1 + b * r2)
    assert np.allclose(lhs, a * out(r1) + b * out(r2), rtol=1e-10, atol=1e-12 * np.abs(lhs).max())
