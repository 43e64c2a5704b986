"""yuzen_b200 -- the implicit time step of Yuzen's well-mixed film-height
equation on one B200 (sm_100a), behind a C ABI (include/yuzen_b200.h).

This module is a thin ctypes binding of that ABI.  It mirrors the reference's
solver seam (yuzen/src/numerics/LinearSolverBackend.h:38-131):

    LinearSolverSettings   -- the settings handed over on every solve
    MakeLinearSolverBackend("b200") -> B200Backend, an ILinearSolverBackend
        with Name / Build / Solve / Memory / SetMemory

The CUDA library libyuzen_b200.so must have been built in-tree
(python -m yuzen_b200.build); there is no CPU fallback, and every entry point
raises when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = [
    "LinearSolverSettings", "B200Backend", "MakeLinearSolverBackend", "CrsPattern",
    "lib", "lib_path", "YzError", "EXPORTED_SYMBOLS", "dot", "spmv", "PREC_FP64", "PREC_FP32_CYCLE", "PREC_FP32_MATRIX",
]

_HERE = Path(__file__).resolve().parent
_LIB = None

#: every symbol include/yuzen_b200.h declares
EXPORTED_SYMBOLS = (
    "yz_last_error", "yz_solver_create", "yz_solver_destroy", "yz_solver_set_pattern",
    "yz_solver_solve", "yz_solver_solve_device", "yz_solver_set_precision",
    "yz_solver_memory", "yz_solver_set_memory", "yz_solver_levels", "yz_solver_level_info",
    "yz_solver_level_copy", "yz_solver_last_timing", "yz_solver_launches", "yz_dot", "yz_spmv",
    "yz_step_create", "yz_step_destroy", "yz_step_advance", "yz_step_get_fields", "yz_step_pattern",
    "yz_step_system", "yz_pattern_2d", "yz_step_set_fields", "yz_launch_count",
    "yz_time_kernel", "yz_kernel_time", "yz_dot_noalloc", "yz_dot_noalloc_max",
    "yz_step_conc_pattern", "yz_step_conc_system", "yz_step_set_precision", "yz_solver_set_amg_reuse",
    "yz_step_set_amg_reuse", "yz_solver_set_graph_loop", "yz_step_set_graph_loop", "yz_step_energy",
    "yz_step_set_energy",
    # the learned preconditioner
    "yz_unet_create", "yz_unet_destroy", "yz_unet_param_count", "yz_unet_get_params", "yz_unet_set_params",
    "yz_unet_forward", "yz_unet_loss_grad", "yz_unet_add_sample", "yz_unet_samples", "yz_unet_get_sample", "yz_unet_train",
    "yz_unet_apply", "yz_solver_set_learned", "yz_solver_set_aux", "yz_solver_learned_stats",
    "yz_step_set_learned", "yz_conv3x3", "yz_fault_inject", "yz_step_state_size", "yz_step_get_state",
    "yz_step_set_state", "yz_profile_enabled", "yz_profile_entry", "yz_profile_reset", "yz_solver_set_tuning",
    "yz_step_set_tuning",
    # the ConcZ model (seam 3)
    "yz_cz_create", "yz_cz_destroy", "yz_cz_advance", "yz_cz_get_fields", "yz_cz_set_fields", "yz_cz_set_precision",
    "yz_cz_set_amg_reuse", "yz_cz_set_tuning", "yz_cz_set_learned", "yz_cz_parts", "yz_cz_read", "yz_cz_pattern", "yz_cz_build_pattern", "yz_exp_cr",
)

#: the preconditioner's arithmetic (YZ_PREC_* of include/yuzen_b200.h)
PREC_FP64 = 0
PREC_FP32_CYCLE = 1
PREC_FP32_MATRIX = 2


class YzError(RuntimeError):
    """A negative status of the C ABI (-1 usage error, -2 CUDA error, -3 a
    failed time step); `status` holds it."""

    def __init__(self, msg: str, status: int = -2):
        super().__init__(msg)
        self.status = status


class StepFailedError(YzError):
    """Status -3: the time step failed numerically where the reference aborts
    with its FatalError (dt below MinDt; no convergence at a fixed step)."""


def lib_path() -> Path:
    return _HERE / "libyuzen_b200.so"


class _Settings(ctypes.Structure):
    _fields_ = [("precondition", ctypes.c_int), ("scaling", ctypes.c_int),
                ("max_iteration", ctypes.c_int), ("epsilon", ctypes.c_double),
                ("conc", ctypes.c_int)]


_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def lib():
    """Load libyuzen_b200.so (built in-tree).  Raises if it was not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = lib_path()
    if not p.exists():
        raise RuntimeError(f"{p} is not built: run `python -m yuzen_b200.build` "
                           "(the library has no CPU fallback)")
    L = ctypes.CDLL(str(p))
    L.yz_last_error.restype = ctypes.c_char_p
    L.yz_solver_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.yz_solver_destroy.argtypes = [ctypes.c_void_p]
    L.yz_solver_set_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p]
    L.yz_solver_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Settings), _f64p, _f64p, _f64p, _i32p, _f64p]
    L.yz_solver_solve_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Settings), ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, _i32p, _f64p]
    L.yz_solver_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_solver_set_amg_reuse.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_solver_set_graph_loop.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_solver_set_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.yz_solver_memory.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int]
    L.yz_solver_set_memory.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int]
    L.yz_solver_levels.argtypes = [ctypes.c_void_p]
    L.yz_solver_level_info.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p, _i32p]
    L.yz_solver_level_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i32p]
    L.yz_solver_last_timing.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_solver_launches.argtypes = [ctypes.c_void_p]
    L.yz_solver_launches.restype = ctypes.c_longlong
    L.yz_dot.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p]
    L.yz_spmv.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
    L.yz_dot_noalloc.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.yz_dot_noalloc_max.restype = ctypes.c_longlong
    L.yz_time_kernel.argtypes = [ctypes.c_char_p]
    L.yz_kernel_time.argtypes = [_f64p, ctypes.POINTER(ctypes.c_longlong)]
    _LIB = L
    return L


def _check(status: int, what: str) -> int:
    if status < 0:
        msg = lib().yz_last_error().decode(errors="replace")
        cls = StepFailedError if status == -3 else YzError
        raise cls(f"{what}: status {status}: {msg}", status)
    return status


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_i32p)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_f64p)


class LinearSolverSettings:
    """LinearSolverSettings (LinearSolverBackend.h:38-51)."""
    tp_None, tp_Jacobi, tp_ILU = 0, 1, 2

    def __init__(self, precondition: int = 2, scaling: bool = True, maxIteration: int = 100,
                 epsilon: float = 1e-12, conc: bool = False):
        self.precondition = precondition
        self.scaling = scaling
        self.maxIteration = maxIteration
        self.epsilon = epsilon
        self.conc = conc

    def _c(self) -> _Settings:
        return _Settings(int(self.precondition), int(bool(self.scaling)), int(self.maxIteration),
                         float(self.epsilon), int(bool(self.conc)))


class CrsPattern:
    """The view of a CRS_Matrix a backend receives (CRS_Matrix.h:242-269):
    row pointers, storage-order columns (diagonal first), the column-sorted
    mirror and the permutation that gathers values into it."""

    def __init__(self, rowptr, col, sorted_col=None, sorted_src=None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        n = self.rowptr.size - 1
        if sorted_col is None or sorted_src is None:
            scol = np.empty_like(self.col)
            ssrc = np.empty_like(self.col)
            for i in range(n):
                st, ed = self.rowptr[i], self.rowptr[i + 1]
                order = np.argsort(self.col[st:ed], kind="stable")
                scol[st:ed] = self.col[st:ed][order]
                ssrc[st:ed] = st + order
            sorted_col, sorted_src = scol, ssrc
        self.sorted_col = np.ascontiguousarray(sorted_col, dtype=np.int32)
        self.sorted_src = np.ascontiguousarray(sorted_src, dtype=np.int32)

    @property
    def n(self) -> int:
        return self.rowptr.size - 1

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])


class B200Backend:
    """ILinearSolverBackend on the device (LinearSolverBackend.h:56-103).

    Solve(settings, pattern, values, rhs, x) -> (ret, iter, resid), x updated
    in place; ret 0 converged, 1 iteration limit, 2 breakdown / NaN."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().yz_solver_create(device, ctypes.byref(self._h)), "yz_solver_create")
        self._pattern = None

    def Name(self) -> str:
        return "b200"

    def Build(self, nRow: int, nonZero: int, nonZL: int = 0, nonZU: int = 0) -> None:
        # storage is sized when the pattern is handed over (SetPattern)
        self._n, self._nnz = nRow, nonZero

    def SetPattern(self, pat: CrsPattern) -> None:
        _check(lib().yz_solver_set_pattern(self._h, pat.n, pat.nnz, _ip(pat.rowptr), _ip(pat.sorted_col),
                                           _ip(pat.sorted_src)), "yz_solver_set_pattern")
        self._pattern = pat     # held, so that the identity test below cannot see a recycled id

    def Solve(self, s: LinearSolverSettings, pat: CrsPattern, values, rhs, x):
        if self._pattern is not pat:
            self.SetPattern(pat)
        values = np.ascontiguousarray(values, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("x must be a contiguous float64 array (it is updated in place)")
        it = ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        c = s._c()
        ret = _check(lib().yz_solver_solve(self._h, ctypes.byref(c), _fp(values), _fp(rhs), _fp(x),
                                           ctypes.byref(it), ctypes.byref(res)), "yz_solver_solve")
        return ret, it.value, res.value

    def SolveDevice(self, s: LinearSolverSettings, values_ptr: int, rhs_ptr: int, x_ptr: int):
        it = ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        c = s._c()
        ret = _check(lib().yz_solver_solve_device(self._h, ctypes.byref(c), ctypes.c_void_p(values_ptr),
                                                  ctypes.c_void_p(rhs_ptr), ctypes.c_void_p(x_ptr),
                                                  ctypes.byref(it), ctypes.byref(res)), "yz_solver_solve_device")
        return ret, it.value, res.value

    def SetPrecision(self, precision: int) -> None:
        """PREC_FP64 (the drop-in path), PREC_FP32_CYCLE (the V-cycle in float
        inside the FP64 BiCGStab) or PREC_FP32_MATRIX (that, and the
        BiCGStab's SpMVs on the matrix rounded to float), from the next solve
        on."""
        _check(lib().yz_solver_set_precision(self._h, precision), "yz_solver_set_precision")

    def SetAmgReuse(self, max_solves: int) -> None:
        """0: a new AMG set-up every solve (the reference's way); k > 0: a
        set-up serves up to k further solves (yz_solver_set_amg_reuse)."""
        _check(lib().yz_solver_set_amg_reuse(self._h, max_solves), "yz_solver_set_amg_reuse")

    def SetGraphLoop(self, on: bool) -> None:
        """The BiCGStab loop as one CUDA graph launch (default) or from the
        stream (yz_solver_set_graph_loop)."""
        _check(lib().yz_solver_set_graph_loop(self._h, int(bool(on))), "yz_solver_set_graph_loop")

    def SetTuning(self, fuse_from: int = -1, coarse_lanes: int = 0, fine_sweeps: int = 0) -> None:
        """The FP32 V-cycle's shape (yz_solver_set_tuning): the first fused
        coarse level (-1 default, 0 none), the coarse levels' lanes a row (0:
        by row length), the finest level's post-smoothing sweeps (0: default)."""
        _check(lib().yz_solver_set_tuning(self._h, int(fuse_from), int(coarse_lanes), int(fine_sweeps)),
               "yz_solver_set_tuning")

    def Memory(self) -> list:
        buf = np.zeros(8, dtype=np.float64)
        k = _check(lib().yz_solver_memory(self._h, _fp(buf), 8), "yz_solver_memory")
        return buf[:k].tolist()

    def SetMemory(self, m) -> None:
        a = np.ascontiguousarray(m, dtype=np.float64)
        _check(lib().yz_solver_set_memory(self._h, _fp(a), a.size), "yz_solver_set_memory")

    def levels(self) -> list:
        """The AMG hierarchy of the last AMG solve: one dict per level."""
        L = lib()
        out = []
        nl = _check(L.yz_solver_levels(self._h), "yz_solver_levels")
        for l in range(nl):
            rows, nnza, nnzp, direct = (ctypes.c_int() for _ in range(4))
            _check(L.yz_solver_level_info(self._h, l, ctypes.byref(rows), ctypes.byref(nnza),
                                          ctypes.byref(nnzp), ctypes.byref(direct)), "level_info")
            n, na, npn = rows.value, nnza.value, nnzp.value
            d = {"rows": n, "nnz_a": na, "nnz_p": npn, "direct": bool(direct.value),
                 "a_ptr": np.zeros(n + 1, np.int32), "a_col": np.zeros(max(na, 1), np.int32),
                 "a_val": np.zeros(max(na, 1)), "p_ptr": np.zeros(n + 1, np.int32),
                 "p_col": np.zeros(max(npn, 1), np.int32), "p_val": np.zeros(max(npn, 1)),
                 "agg": np.full(n, -1, np.int32)}
            _check(L.yz_solver_level_copy(self._h, l, _ip(d["a_ptr"]), _ip(d["a_col"]), _fp(d["a_val"]),
                                          _ip(d["p_ptr"]), _ip(d["p_col"]), _fp(d["p_val"]), _ip(d["agg"])),
                   "level_copy")
            d["a_col"], d["a_val"] = d["a_col"][:na], d["a_val"][:na]
            d["p_col"], d["p_val"] = d["p_col"][:npn], d["p_val"][:npn]
            out.append(d)
        return out

    def last_timing(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().yz_solver_last_timing(self._h, ctypes.byref(a), ctypes.byref(b)), "last_timing")
        return a.value, b.value

    def launches(self) -> int:
        return int(lib().yz_solver_launches(self._h))

    def SetLearned(self, net, mode: int, collect_solves: int = 0, per_solve: int = 0, cap_factor: float = 1.0):
        """The learned preconditioner (yuzen_b200.learned.UNet) of the film's
        solves: mode 0 off, 1 collect (AMG solves feed its sample ring), 2 use
        (flexible BiCGStab with the network first, SA-AMG the fallback)."""
        from . import learned
        L = learned._bind()
        self._net = net
        _check(L.yz_solver_set_learned(self._h, net.handle if net is not None else None, mode, collect_solves,
                                       per_solve, cap_factor), "yz_solver_set_learned")

    def SetAux(self, h_ptr: int | None) -> None:
        """The film height on the device (a pointer to n doubles) the network
        reads as a feature; None: none."""
        from . import learned
        _check(learned._bind().yz_solver_set_aux(self._h, ctypes.c_void_p(h_ptr) if h_ptr else None),
               "yz_solver_set_aux")

    def learned_stats(self) -> dict:
        from . import learned
        v = [ctypes.c_int() for _ in range(4)]
        _check(learned._bind().yz_solver_learned_stats(self._h, *[ctypes.byref(x) for x in v]), "learned_stats")
        return dict(zip(("solves", "fallbacks", "iterations", "skipped"), (x.value for x in v)))

    def close(self) -> None:
        if self._h:
            lib().yz_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def MakeLinearSolverBackend(name: str, inPlane: int = 2, device: int = 0) -> B200Backend:
    """The factory entry for the name this library adds ("b200")."""
    if name != "b200":
        raise ValueError(f"this library provides the backend 'b200', not {name!r}")
    return B200Backend(device)


def dot(x, y) -> float:
    """The deterministic dot product of the solve, on the device."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    out = ctypes.c_double()
    _check(lib().yz_dot(x.size, _fp(x), _fp(y), ctypes.byref(out)), "yz_dot")
    return out.value


def spmv(rowptr, col, val, x) -> np.ndarray:
    """CRS_Matrix::MatVec on the device: y_i summed from 0.0 in stored order."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(rowptr.size - 1)
    _check(lib().yz_spmv(rowptr.size - 1, int(rowptr[-1]), _ip(rowptr), _ip(col), _fp(val), _fp(x), _fp(y)),
           "yz_spmv")
    return y


def time_kernel(name: str | None) -> None:
    """Bracket every later launch of the named kernel with CUDA events."""
    _check(lib().yz_time_kernel(name.encode() if name else None), "yz_time_kernel")


def kernel_time():
    """(total device ms, launches) of the kernel selected by time_kernel()."""
    ms = ctypes.c_double()
    cnt = ctypes.c_longlong()
    _check(lib().yz_kernel_time(ctypes.byref(ms), ctypes.byref(cnt)), "yz_kernel_time")
    return ms.value, cnt.value


def dot_noalloc(n: int, x_ptr: int, y_ptr: int, out_ptr: int, stream: int = 0) -> None:
    """yz_dot_noalloc on device pointers (the caller owns every buffer)."""
    _check(lib().yz_dot_noalloc(int(n), ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), ctypes.c_void_p(out_ptr),
                                ctypes.c_void_p(stream) if stream else None), "yz_dot_noalloc")


def fault_inject(at: int, count: int = 1) -> None:
    """The reference's fault switch (YUZEN_FAULT_AMGCL=at:count): `count`
    solves of the process from the at-th that reaches the SA-AMG / Jacobi path
    break down before iterating; at = 0 off (yz_fault_inject)."""
    L = lib()
    L.yz_fault_inject.argtypes = [ctypes.c_longlong, ctypes.c_longlong]
    _check(L.yz_fault_inject(at, count), "yz_fault_inject")


def profile_table() -> dict:
    """The profile table (yz_profile_entry): {name: (calls, device seconds)}
    of every scope run so far; empty unless YUZEN_PROFILE was set when the
    process first opened one."""
    L = lib()
    L.yz_profile_entry.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_longlong),
                                   ctypes.POINTER(ctypes.c_double)]
    out = {}
    i = 0
    while True:
        name, calls, sec = ctypes.c_char_p(), ctypes.c_longlong(), ctypes.c_double()
        r = L.yz_profile_entry(i, ctypes.byref(name), ctypes.byref(calls), ctypes.byref(sec))
        _check(r, "yz_profile_entry")
        if r == 1:
            return out
        out[name.value.decode()] = (calls.value, sec.value)
        i += 1


def profile_reset() -> None:
    """Zero the profile table's totals (yz_profile_reset)."""
    _check(lib().yz_profile_reset(), "yz_profile_reset")
