"""ctypes binding of the learned preconditioner (include/yuzen_b200.h,
yz_unet_* and the learned settings of the solver and the step).

    net = UNet(nx, ny, capacity=64, seed=1)
    net.add_sample(r, z, diag, h)          # (residual, V-cycle answer) pairs
    loss, val = net.train(200, batch=4, lr=1e-3, holdout=4)
    backend.SetLearned(net, mode=2)        # the flexible BiCGStab tries it first

The network is the device's (yuzen_b200/csrc/yz_unet.cu); there is no CPU
path here.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _check, _fp, _ip, lib

_f32p = ctypes.POINTER(ctypes.c_float)
_BOUND = False


class LearnedConfig(ctypes.Structure):
    """yz_learned_cfg: the step's learned preconditioner."""
    _fields_ = [("collect_solves", ctypes.c_int), ("samples_per_solve", ctypes.c_int), ("capacity", ctypes.c_int),
                ("train_iters", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_float),
                ("holdout", ctypes.c_int), ("cap_factor", ctypes.c_double), ("seed", ctypes.c_uint),
                ("activation", ctypes.c_int)]


def default_config(**over) -> LearnedConfig:
    d = {"collect_solves": 6, "samples_per_solve": 8, "capacity": 48, "train_iters": 300, "batch": 4,
         "lr": 1e-3, "holdout": 4, "cap_factor": 1.0, "seed": 1, "activation": 0}
    d.update(over)
    return LearnedConfig(**d)


def _bind():
    global _BOUND
    L = lib()
    if _BOUND:
        return L
    vp = ctypes.c_void_p
    L.yz_unet_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                                 ctypes.POINTER(vp)]
    L.yz_unet_destroy.argtypes = [vp]
    L.yz_unet_param_count.argtypes = [vp]
    L.yz_unet_param_count.restype = ctypes.c_longlong
    L.yz_unet_get_params.argtypes = [vp, _f32p]
    L.yz_unet_set_params.argtypes = [vp, _f32p]
    L.yz_unet_forward.argtypes = [vp, _f32p, _f32p]
    L.yz_unet_loss_grad.argtypes = [vp, _f32p, _f32p, ctypes.POINTER(ctypes.c_double), _f32p]
    L.yz_unet_add_sample.argtypes = [vp] + [ctypes.POINTER(ctypes.c_double)] * 4
    L.yz_unet_samples.argtypes = [vp]
    L.yz_unet_get_sample.argtypes = [vp, ctypes.c_int, _f32p, ctypes.POINTER(ctypes.c_int)]
    L.yz_unet_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.yz_unet_apply.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.yz_solver_set_learned.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    L.yz_solver_set_aux.argtypes = [vp, vp]
    L.yz_solver_learned_stats.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 4
    L.yz_step_set_learned.argtypes = [vp, ctypes.POINTER(LearnedConfig)]
    L.yz_cz_set_learned.argtypes = [vp, ctypes.POINTER(LearnedConfig)]
    L.yz_conv3x3.argtypes = [ctypes.c_int] * 7 + [_f32p, _f32p, _f32p, _f32p]
    _BOUND = True
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class UNet:
    """The device network of one grid (nx x ny points, ghosts included)."""

    def __init__(self, nx: int, ny: int, capacity: int = 64, seed: int = 1, activation: int = 0, device: int = 0):
        L = _bind()
        self.nx, self.ny, self.n = nx, ny, nx * ny
        self.activation = activation
        self._h = ctypes.c_void_p()
        _check(L.yz_unet_create(device, nx, ny, capacity, seed, activation, ctypes.byref(self._h)), "yz_unet_create")

    @property
    def handle(self):
        return self._h

    def param_count(self) -> int:
        return int(lib().yz_unet_param_count(self._h))

    def params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        _check(lib().yz_unet_get_params(self._h, out.ctypes.data_as(_f32p)), "yz_unet_get_params")
        return out

    def set_params(self, p) -> None:
        p = _f32(p)
        if p.size != self.param_count():
            raise ValueError("wrong parameter count")
        _check(lib().yz_unet_set_params(self._h, p.ctypes.data_as(_f32p)), "yz_unet_set_params")

    def forward(self, feat3) -> np.ndarray:
        f = _f32(feat3).reshape(-1)
        if f.size != 3 * self.n:
            raise ValueError("feat3 needs 3 x n values")
        out = np.zeros(self.n, np.float32)
        _check(lib().yz_unet_forward(self._h, f.ctypes.data_as(_f32p), out.ctypes.data_as(_f32p)), "yz_unet_forward")
        return out

    def loss_grad(self, feat3, target):
        f = _f32(feat3).reshape(-1)
        t = _f32(target)
        g = np.zeros(self.param_count(), np.float32)
        loss = ctypes.c_double()
        _check(lib().yz_unet_loss_grad(self._h, f.ctypes.data_as(_f32p), t.ctypes.data_as(_f32p), ctypes.byref(loss),
                                       g.ctypes.data_as(_f32p)), "yz_unet_loss_grad")
        return loss.value, g

    def add_sample(self, r, z, diag, h=None) -> None:
        r, z, d = (np.ascontiguousarray(a, np.float64) for a in (r, z, diag))
        hh = np.ascontiguousarray(h, np.float64) if h is not None else None
        _check(lib().yz_unet_add_sample(self._h, _fp(r), _fp(z), _fp(d), _fp(hh) if hh is not None else None),
               "yz_unet_add_sample")

    def samples(self) -> int:
        return int(lib().yz_unet_samples(self._h))

    def sample(self, k: int) -> dict:
        """Slot k of the pair ring: r and z scaled by 1/rms(r), the two
        feature maps it was stored with, and whether the slot holds a pair."""
        out = np.zeros(4 * self.n, np.float32)
        valid = ctypes.c_int()
        _check(lib().yz_unet_get_sample(self._h, int(k), out.ctypes.data_as(_f32p), ctypes.byref(valid)),
               "yz_unet_get_sample")
        r, z, f1, f2 = out.reshape(4, self.n)
        return {"r": r, "z": z, "f1": f1, "f2": f2, "valid": bool(valid.value)}

    def train(self, iters: int, batch: int = 4, lr: float = 1e-3, holdout: int = 0):
        loss, val = ctypes.c_double(), ctypes.c_double()
        _check(lib().yz_unet_train(self._h, iters, batch, lr, holdout, ctypes.byref(loss), ctypes.byref(val)),
               "yz_unet_train")
        return loss.value, val.value

    def close(self) -> None:
        if self._h:
            lib().yz_unet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def features(r, diag, h=None):
    """The three normalised maps the network's inputs are formed from
    (float32, 3 x n): r / rms(r), log10 |diag| / 4, log10 h / 2 + 1 (0
    without h) -- as the device forms them (yz_learned.h)."""
    r = np.asarray(r, np.float64)
    rms = np.sqrt(np.sum(r * r) / r.size)
    f = np.zeros((3, r.size), np.float32)
    f[0] = (r.astype(np.float32) * np.float32(1.0 / rms if rms > 0 else 0.0))
    f[1] = np.log10(np.maximum(np.abs(diag), 1e-30)) * 0.25
    if h is not None:
        f[2] = np.log10(np.maximum(h, 1e-30)) * 0.5 + 1.0
    return f, rms


def conv3x3(x, w, bias, real_w: int, real_h: int, relu: bool) -> np.ndarray:
    """One convolution of the network's tensor-core kernel: x (H, W, cin),
    w (n, 9, cin), bias (n,) or None; returns (H, W, n) float32."""
    L = _bind()
    x = _f32(x)
    H, W, cin = x.shape
    w = _f32(w)
    n = w.shape[0]
    b = _f32(bias) if bias is not None else None
    y = np.zeros((H, W, n), np.float32)
    _check(L.yz_conv3x3(H, W, cin, n, real_w, real_h, int(bool(relu)), x.ctypes.data_as(_f32p), w.ctypes.data_as(_f32p),
                        b.ctypes.data_as(_f32p) if b is not None else None, y.ctypes.data_as(_f32p)), "yz_conv3x3")
    return y


def _main() -> None:
    """python -m yuzen_b200.learned NX: the network on an NX x NX grid with
    random inputs -- two forward passes and two loss-and-gradient passes (the
    launch sequence of one application and of one training sample) -- and
    their host-clock times."""
    import sys
    import time
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 516
    net = UNet(n, n, capacity=4, seed=1)
    rng = np.random.default_rng(0)
    f = rng.standard_normal((3, n * n)).astype(np.float32)
    t = rng.standard_normal(n * n).astype(np.float32)
    for name, fn in (("forward", lambda: net.forward(f)), ("loss and gradient", lambda: net.loss_grad(f, t))):
        for k in range(2):
            t0 = time.perf_counter()
            fn()
            print(f"{name} {k}: {1e3 * (time.perf_counter() - t0):.2f} ms (host clock, copies included)")


if __name__ == "__main__":
    _main()
