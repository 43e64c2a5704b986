"""CPU restatement of the learned preconditioner's network (TEST INFRASTRUCTURE).

This is the checker the device network (yuzen_b200/csrc/yz_unet.cu) is
compared against; nothing of the product path imports it.  The reference has
no learned preconditioner, so this module restates the device network's own
definition (yuzen_b200/csrc/yz_learned.h): the image geometry, the input
channels (r and its products with the two feature maps f1, f2: r, r f1,
r f2, r f1^2, r f2^2, r f1 f2), the U-Net (levels of 16, 32, 64, 64
channels; 3x3 convolutions, with bias and ReLU when act = 1, neither when
act = 0; 2x2 average pooling; nearest upsampling with the encoder's output
concatenated in front; a 1x1 output layer), the loss sum (out - t)^2 / n
over the real pixels, and the analytic gradient of that loss w.r.t. every
weight (the biases' gradients are 0 when act = 0: the device keeps them
at 0).

Numbers are float64.  With bf16=True every tensor the device stores in BF16
(activations, the gradients of activations, the network's inputs and packed
weights) is rounded to BF16 (round to nearest even) at the same points, so the
device's results differ from this only by its FP32 accumulation order; with
bf16=False it is the exact float64 network, which the finite-difference test
pins.  The parameter vector has the device's order: per convolution (enc0,
enc1, enc2, bott, dec2, dec1, dec0) W[cout][9][cin] then b[cout], then the
output layer's 16 weights and its bias.
"""
from __future__ import annotations

import numpy as np

#  (cin, cout, level) of the seven 3x3 convolutions, in parameter order
CONVS = [(16, 16, 0), (16, 32, 1), (32, 64, 2), (64, 64, 3), (128, 64, 2), (96, 32, 1), (48, 16, 0)]
ENC0, ENC1, ENC2, BOTT, DEC2, DEC1, DEC0 = range(7)


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def geometry(nx: int, ny: int) -> list:
    """Per level (H, W, realH, realW): W_0 = 8 (ceil(nx/8) + 1) (at least one
    zero column right of the real region at every level), H_0 = 8 ceil(ny/8),
    halved per level; the real region halves rounding up."""
    lv = [(8 * ((ny + 7) // 8), 8 * ((nx + 7) // 8 + 1), ny, nx)]
    for _ in range(3):
        H, W, rh, rw = lv[-1]
        lv.append((H // 2, W // 2, (rh + 1) // 2, (rw + 1) // 2))
    return lv


def param_layout():
    out, off = [], 0
    for cin, cout, _ in CONVS:
        out.append((off, off + 9 * cin * cout))
        off += 9 * cin * cout + cout
    return out, off, off + 16


def param_count() -> int:
    return param_layout()[2] + 1


def unpack(params: np.ndarray):
    lay, ow, ob = param_layout()
    Ws, bs = [], []
    for (wo, bo), (cin, cout, _) in zip(lay, CONVS):
        Ws.append(params[wo:bo].reshape(cout, 9, cin).astype(np.float64))
        bs.append(params[bo:bo + cout].astype(np.float64))
    return Ws, bs, params[ow:ow + 16].astype(np.float64), float(params[ob])


class Net:
    def __init__(self, nx: int, ny: int, bf16: bool = True, act: int = 1):
        self.nx, self.ny, self.n = nx, ny, nx * ny
        self.lv = geometry(nx, ny)
        self.bf16 = bf16
        self.act = act

    def r(self, x):
        return to_bf16(x) if self.bf16 else np.asarray(x, dtype=np.float64)

    # ------------------------------------------------------------------
    def real(self, l):
        H, W, rh, rw = self.lv[l]
        m = np.zeros((H, W), dtype=bool)
        m[:rh, :rw] = True
        return m.reshape(-1)

    def shifted(self, x, l, tap):
        """x[p + dy W + dx] over the linear pixel index (0 outside the image)."""
        H, W, _, _ = self.lv[l]
        dy, dx = tap // 3 - 1, tap % 3 - 1
        s = dy * W + dx
        out = np.zeros_like(x)
        HW = H * W
        if s >= 0:
            out[:HW - s] = x[s:]
        else:
            out[-s:] = x[:HW + s]
        return out

    def conv(self, x, Wt, b, l, relu):
        """x: (HW, cin); Wt: (cout, 9, cin); returns the stored (rounded) output."""
        acc = np.zeros((x.shape[0], Wt.shape[0]))
        for t in range(9):
            acc += self.shifted(x, l, t) @ Wt[:, t, :].T
        if b is not None:
            acc += b
        if relu:
            acc = np.maximum(acc, 0.0)
        acc[~self.real(l)] = 0.0
        return self.r(acc)

    def conv_t(self, g, Wt, l):
        """the transposed convolution: dx[q] = sum_tap g[q - off(tap)] W[:, tap, :]"""
        acc = np.zeros((g.shape[0], Wt.shape[2]))
        for t in range(9):
            acc += self.shifted(g, l, 8 - t) @ Wt[:, t, :]
        acc[~self.real(l)] = 0.0
        return self.r(acc)

    def wgrad(self, x, g, l):
        """dW[n][tap][ci] = sum_p g[p][n] x[p + off(tap)][ci]; db[n] = sum_p g[p][n]"""
        dW = np.zeros((g.shape[1], 9, x.shape[1]))
        for t in range(9):
            dW[:, t, :] = g.T @ self.shifted(x, l, t)
        return dW, g.sum(axis=0)

    def pool(self, x, l):
        H, W, _, _ = self.lv[l]
        Hl, Wl, _, _ = self.lv[l + 1]
        C = x.shape[1]
        a = x.reshape(H, W, C)
        o = 0.25 * (a[0::2, 0::2] + a[0::2, 1::2] + a[1::2, 0::2] + a[1::2, 1::2])
        o = o.reshape(Hl * Wl, C)
        o[~self.real(l + 1)] = 0.0
        return self.r(o)

    def up(self, x, l):
        """x at level l+1 to level l (nearest), 0 outside the real region"""
        H, W, _, _ = self.lv[l]
        Hl, Wl, _, _ = self.lv[l + 1]
        C = x.shape[1]
        a = x.reshape(Hl, Wl, C)
        o = np.repeat(np.repeat(a, 2, axis=0), 2, axis=1).reshape(H * W, C)
        o[~self.real(l)] = 0.0
        return o

    def up_back(self, g, l):
        """the sum of a level-l gradient over the four children of each level-(l+1) pixel (real children only)"""
        H, W, _, _ = self.lv[l]
        Hl, Wl, _, _ = self.lv[l + 1]
        C = g.shape[1]
        gg = g.copy()
        gg[~self.real(l)] = 0.0
        a = gg.reshape(H, W, C)
        o = a[0::2, 0::2] + a[0::2, 1::2] + a[1::2, 0::2] + a[1::2, 1::2]
        o = o.reshape(Hl * Wl, C)
        o[~self.real(l + 1)] = 0.0
        return o

    # ------------------------------------------------------------------
    def image(self, feat3):
        """the input image (H0 W0, 16): channels r, r f1, r f2, r f1^2,
        r f2^2, r f1 f2 of the maps feat3 = (r, f1, f2), products in float32
        as the device forms them, bf16"""
        H, W, _, _ = self.lv[0]
        F = np.zeros((H * W, 16))
        idx = self.rows_to_pixels()
        r, f1, f2 = (np.asarray(feat3[c], dtype=np.float32) for c in range(3))
        if not self.bf16:
            r, f1, f2 = (np.asarray(feat3[c], dtype=np.float64) for c in range(3))
        for c, v in enumerate((r, r * f1, r * f2, (r * f1) * f1, (r * f2) * f2, (r * f1) * f2)):
            F[idx, c] = v
        return self.r(F)

    def rows_to_pixels(self):
        i = np.arange(self.n)
        return (i // self.nx) * self.lv[0][1] + (i % self.nx)

    def forward(self, params, feat3):
        Ws, bs, wo, bo = unpack(params)
        if self.bf16:
            Ws = [to_bf16(w) for w in Ws]
        a = {}
        F = self.image(feat3)
        a["F"] = F
        A = self.act == 1
        E0 = self.conv(F, Ws[ENC0], bs[ENC0], 0, A)
        P1 = self.pool(E0, 0)
        E1 = self.conv(P1, Ws[ENC1], bs[ENC1], 1, A)
        P2 = self.pool(E1, 1)
        E2 = self.conv(P2, Ws[ENC2], bs[ENC2], 2, A)
        P3 = self.pool(E2, 2)
        B3 = self.conv(P3, Ws[BOTT], bs[BOTT], 3, A)
        U2 = np.concatenate([E2, self.up(B3, 2)], axis=1)
        D2 = self.conv(U2, Ws[DEC2], bs[DEC2], 2, A)
        U1 = np.concatenate([E1, self.up(D2, 1)], axis=1)
        D1 = self.conv(U1, Ws[DEC1], bs[DEC1], 1, A)
        U0 = np.concatenate([E0, self.up(D1, 0)], axis=1)
        D0 = self.conv(U0, Ws[DEC0], bs[DEC0], 0, A)
        a.update(E0=E0, P1=P1, E1=E1, P2=P2, E2=E2, P3=P3, B3=B3, U2=U2, D2=D2, U1=U1, D1=D1, U0=U0, D0=D0, W=Ws,
                 wo=wo, bo=bo)
        out = D0[self.rows_to_pixels()] @ wo + bo
        return out, a

    def loss_grad(self, params, feat3, target):
        """(loss, gradient w.r.t. params) for one pair (feat3: 3 x n, target: n)"""
        out, a = self.forward(params, feat3)
        n = self.n
        diff = out - target
        loss = float(np.sum(diff * diff) / n)
        g = 2.0 * diff / n
        Ws, wo = a["W"], a["wo"]
        lay, ow, ob = param_layout()
        grad = np.zeros(param_count())
        pix = self.rows_to_pixels()
        D0 = a["D0"]
        grad[ow:ow + 16] = g @ D0[pix]
        grad[ob] = g.sum() if self.act else 0.0
        gD0 = np.zeros_like(D0)
        gD0[pix] = np.outer(g, wo) * ((D0[pix] > 0) if self.act else 1.0)
        gD0 = self.r(gD0)

        def put(k, dW, db):
            wo_, bo_ = lay[k]
            grad[wo_:bo_] += dW.reshape(-1)
            if self.act:
                grad[bo_:bo_ + CONVS[k][1]] += db

        def mask(x):
            return (x > 0) if self.act else 1.0

        # dec0
        gU0 = self.conv_t(gD0, Ws[DEC0], 0)
        put(DEC0, *self.wgrad(a["U0"], gD0, 0))
        gD1 = self.r(self.up_back(gU0[:, 16:48], 0) * mask(a["D1"]))
        # dec1
        gU1 = self.conv_t(gD1, Ws[DEC1], 1)
        put(DEC1, *self.wgrad(a["U1"], gD1, 1))
        gD2 = self.r(self.up_back(gU1[:, 32:96], 1) * mask(a["D2"]))
        # dec2
        gU2 = self.conv_t(gD2, Ws[DEC2], 2)
        put(DEC2, *self.wgrad(a["U2"], gD2, 2))
        gB3 = self.r(self.up_back(gU2[:, 64:128], 2) * mask(a["B3"]))
        # bottleneck
        gP3 = self.conv_t(gB3, Ws[BOTT], 3)
        put(BOTT, *self.wgrad(a["P3"], gB3, 3))
        # enc2, enc1, enc0: the skip gradient plus a quarter of the pooled one
        gE2 = self.r(self.skip_back(gU2[:, 0:64], gP3, a["E2"], 2))
        gP2 = self.conv_t(gE2, Ws[ENC2], 2)
        put(ENC2, *self.wgrad(a["P2"], gE2, 2))
        gE1 = self.r(self.skip_back(gU1[:, 0:32], gP2, a["E1"], 1))
        gP1 = self.conv_t(gE1, Ws[ENC1], 1)
        put(ENC1, *self.wgrad(a["P1"], gE1, 1))
        gE0 = self.r(self.skip_back(gU0[:, 0:16], gP1, a["E0"], 0))
        put(ENC0, *self.wgrad(a["F"], gE0, 0))
        return loss, grad

    def skip_back(self, gU, gP, E, l):
        H, W, _, _ = self.lv[l]
        par = self.up(gP, l)
        o = (gU + 0.25 * par) * ((E > 0) if self.act else 1.0)
        o[~self.real(l)] = 0.0
        return o


def init_params(seed: int = 0, act: int = 1) -> np.ndarray:
    """A random draw in the device's parameter order (for the tests; the
    device draws its own from its generator): He-normal weights, small
    biases with act = 1; weights of variance 1/fan-in and zero biases with
    act = 0."""
    rng = np.random.default_rng(seed)
    lay, ow, ob = param_layout()
    p = np.zeros(param_count())
    for (wo, bo), (cin, cout, _) in zip(lay, CONVS):
        p[wo:bo] = rng.normal(0.0, np.sqrt((2.0 if act else 1.0) / (9 * cin)), bo - wo)
        if act:
            p[bo:bo + cout] = rng.normal(0.0, 0.05, cout)
    p[ow:ow + 16] = rng.normal(0.0, 0.25, 16)
    p[ob] = 0.01 if act else 0.0
    return p
