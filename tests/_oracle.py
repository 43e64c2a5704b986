"""ctypes binding of the CPU oracle of the linear solve (oracle/lib/
liboracle_solver.so, built from oracle/solver/yzo_solver.cpp).  Test
infrastructure only: the checker the CUDA library is compared against."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
LIB = REPO / "oracle" / "lib" / "liboracle_solver.so"
REF_TESTS = REPO / "oracle" / "_ref" / "yuzen_tests"
REF_BIN = REPO / "oracle" / "_ref" / "yuzen_oracle"

YZO_AMG, YZO_ILU0 = 0, 1
_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_L = None


class Settings(ctypes.Structure):
    _fields_ = [("precondition", ctypes.c_int), ("scaling", ctypes.c_int),
                ("max_iteration", ctypes.c_int), ("epsilon", ctypes.c_double),
                ("conc", ctypes.c_int)]


def lib():
    global _L
    if _L is not None:
        return _L
    if not LIB.exists():
        subprocess.run(["make", "-C", str(REPO / "oracle"), "solver"], check=True, capture_output=True)
    L = ctypes.CDLL(str(LIB))
    L.yzo_create.restype = ctypes.c_void_p
    L.yzo_create.argtypes = [ctypes.c_int]
    L.yzo_destroy.argtypes = [ctypes.c_void_p]
    L.yzo_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(Settings), ctypes.c_int, _i32p, _i32p, _i32p,
                            _f64p, _f64p, _f64p, _i32p, _f64p]
    L.yzo_memory.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int]
    L.yzo_set_memory.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int]
    L.yzo_levels.argtypes = [ctypes.c_void_p]
    L.yzo_level_info.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p, _i32p]
    L.yzo_level_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i32p]
    L.yzo_dot.restype = ctypes.c_double
    L.yzo_dot.argtypes = [ctypes.c_int, _f64p, _f64p]
    L.yzo_spmv.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
    L.yzo_fault_inject.argtypes = [ctypes.c_long, ctypes.c_long]
    _L = L
    return L


def _ip(a):
    return a.ctypes.data_as(_i32p)


def _fp(a):
    return a.ctypes.data_as(_f64p)


class OracleSolver:
    def __init__(self, flavour: int = YZO_AMG):
        self.h = lib().yzo_create(flavour)

    def solve(self, d: dict, precondition=None, scaling=None, max_iteration=None, epsilon=None, conc=None, x0=None):
        """Solve the system of a dump dict; returns (ret, iter, resid, x)."""
        s = Settings(int(d["precondition"] if precondition is None else precondition),
                     int(d["scaling"] if scaling is None else scaling),
                     int(d["max_iteration"] if max_iteration is None else max_iteration),
                     float(d["epsilon"] if epsilon is None else epsilon),
                     int(d["conc"] if conc is None else conc))
        rowptr = np.ascontiguousarray(d["rowptr"], np.int32)
        scol = np.ascontiguousarray(d["sorted_col"], np.int32)
        ssrc = np.ascontiguousarray(d["sorted_src"], np.int32)
        vals = np.ascontiguousarray(d["values"], np.float64)
        rhs = np.ascontiguousarray(d["rhs"], np.float64)
        x = np.array(d["x0"] if x0 is None else x0, dtype=np.float64, copy=True)
        it = ctypes.c_int()
        res = ctypes.c_double()
        ret = lib().yzo_solve(self.h, ctypes.byref(s), rowptr.size - 1, _ip(rowptr), _ip(scol), _ip(ssrc),
                              _fp(vals), _fp(rhs), _fp(x), ctypes.byref(it), ctypes.byref(res))
        return ret, it.value, res.value, x

    def memory(self):
        buf = np.zeros(8)
        k = lib().yzo_memory(self.h, _fp(buf), 8)
        return buf[:k].tolist()

    def levels(self) -> list:
        L = lib()
        out = []
        for l in range(L.yzo_levels(self.h)):
            rows, nnza, nnzp, direct = (ctypes.c_int() for _ in range(4))
            L.yzo_level_info(self.h, l, ctypes.byref(rows), ctypes.byref(nnza), ctypes.byref(nnzp), ctypes.byref(direct))
            n, na, npn = rows.value, nnza.value, nnzp.value
            d = {"rows": n, "nnz_a": na, "nnz_p": npn, "direct": bool(direct.value),
                 "a_ptr": np.zeros(n + 1, np.int32), "a_col": np.zeros(max(na, 1), np.int32),
                 "a_val": np.zeros(max(na, 1)), "p_ptr": np.zeros(n + 1, np.int32),
                 "p_col": np.zeros(max(npn, 1), np.int32), "p_val": np.zeros(max(npn, 1)),
                 "agg": np.full(n, -1, np.int32)}
            L.yzo_level_copy(self.h, l, _ip(d["a_ptr"]), _ip(d["a_col"]), _fp(d["a_val"]), _ip(d["p_ptr"]),
                             _ip(d["p_col"]), _fp(d["p_val"]), _ip(d["agg"]))
            d["a_col"], d["a_val"] = d["a_col"][:na], d["a_val"][:na]
            d["p_col"], d["p_val"] = d["p_col"][:npn], d["p_val"][:npn]
            out.append(d)
        return out

    def __del__(self):
        try:
            lib().yzo_destroy(self.h)
        except Exception:
            pass


def dot(x, y) -> float:
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    return lib().yzo_dot(x.size, _fp(x), _fp(y))


def spmv(rowptr, col, val, x):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(rowptr.size - 1)
    lib().yzo_spmv(rowptr.size - 1, _ip(rowptr), _ip(col), _fp(val), _fp(x), _fp(y))
    return y


def fault_inject(at: int, count: int = 1) -> None:
    """The oracle's copy of the reference's YUZEN_FAULT_AMGCL switch."""
    lib().yzo_fault_inject(at, count)
