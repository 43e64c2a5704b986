"""ctypes binding of the ConcZ seam of include/yuzen_b200.h (yz_cz_*): the
time step of the ConcZ model -- the semi-implicit film of
CZ_HeightEquation_2D and the concentration through the film of
CZ_ConcEquation_2D (model/ConcZ/CZ2D/) -- on the device, in the reference's
non-dimensional variables.

    p = cz.params_from_record(rec)           # the reference's set-up, as
    m = cz.CzModel(p, rec["xc"], rec["xf"],  # oracle/probe/yz_probe_cz writes it
                   rec["yc"], rec["yf"], rec["h0"], rec["s"], rec["c0"])
    stats = m.advance(5)
    h, c = m.fields()

Arrays: h and s are nx*ny (row jy*nx + ix), c is nx*ny*nz (kz*nx*ny +
jy*nx + ix), ghost layers included."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _Settings, _check, _fp, _ip, lib

_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)


class CzParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("bc", ctypes.c_int * 4),
        ("on_lap", ctypes.c_int), ("on_sc", ctypes.c_int), ("on_vg", ctypes.c_int), ("on_hg", ctypes.c_int),
        ("on_cf", ctypes.c_int), ("on_evap", ctypes.c_int),
        ("ev_conc", ctypes.c_int), ("ev_spatial", ctypes.c_int), ("ev_hast", ctypes.c_int),
        ("dt_control", ctypes.c_int), ("dt_keep_steps", ctypes.c_int), ("c_scheme", ctypes.c_int),
        ("h_lin", _Settings), ("c_lin", _Settings),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dzeta", ctypes.c_double),
        ("theta_h", ctypes.c_double), ("theta_c", ctypes.c_double),
        ("dt", ctypes.c_double), ("dt_old", ctypes.c_double), ("dt_max", ctypes.c_double),
        ("dt_min", ctypes.c_double), ("time", ctypes.c_double),
        ("dt_change_factor", ctypes.c_double), ("dt_criterion", ctypes.c_double),
        ("dt_scale_floor", ctypes.c_double),
        ("As", ctypes.c_double), ("Ma", ctypes.c_double), ("Bo", ctypes.c_double), ("Pgx", ctypes.c_double),
        ("Pgy", ctypes.c_double), ("Sp", ctypes.c_double), ("Df", ctypes.c_double), ("Ev", ctypes.c_double),
        ("rot_center", ctypes.c_double * 2),
        ("visc_c0", ctypes.c_double), ("visc_base", ctypes.c_double), ("visc_exp", ctypes.c_double),
        ("sig_c0", ctypes.c_double), ("sig_base", ctypes.c_double), ("sig_coef", ctypes.c_double),
        ("diff_c0", ctypes.c_double), ("diff_base", ctypes.c_double), ("diff_exp", ctypes.c_double),
        ("ev_mr", ctypes.c_double), ("ev_ms", ctypes.c_double), ("ev_pown", ctypes.c_double),
        ("ev_concr", ctypes.c_double), ("ev_negexp", ctypes.c_double), ("ev_negrmax", ctypes.c_double),
        ("ev_hast_h", ctypes.c_double), ("ev_dr", ctypes.c_double),
        ("coupling_floor", ctypes.c_double),
    ]


class CzStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int), ("linear_iterations", ctypes.c_int), ("conc_iterations", ctypes.c_int),
        ("coupling_passes", ctypes.c_int), ("retries", ctypes.c_int), ("solves", ctypes.c_int),
        ("time", ctypes.c_double), ("dt", ctypes.c_double), ("device_ms", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("learned_solves", ctypes.c_int), ("learned_fallbacks", ctypes.c_int), ("learned_iterations", ctypes.c_int),
        ("learned_samples", ctypes.c_int), ("learned_train_ms", ctypes.c_double), ("learned_val_err", ctypes.c_double),
        ("learned_loss", ctypes.c_double),
    ]


def _bind():
    L = lib()
    if getattr(L, "_cz_bound", False):
        return L
    L.yz_cz_create.argtypes = [ctypes.c_int, ctypes.POINTER(CzParams)] + [_f64p] * 7 + [ctypes.POINTER(ctypes.c_void_p)]
    L.yz_cz_destroy.argtypes = [ctypes.c_void_p]
    L.yz_cz_advance.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(CzStats)]
    L.yz_cz_get_fields.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_cz_set_fields.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_cz_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_cz_set_amg_reuse.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_cz_set_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.yz_cz_parts.argtypes = [ctypes.c_void_p]
    L.yz_cz_read.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _f64p, ctypes.c_longlong]
    L.yz_cz_read.restype = ctypes.c_longlong
    L.yz_cz_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p]
    L.yz_cz_build_pattern.argtypes = [ctypes.POINTER(CzParams), ctypes.c_int, _i32p, _i32p, _i32p]
    L._cz_bound = True
    return L


def _settings(v, eps: float) -> _Settings:
    s = _Settings()
    s.precondition, s.scaling, s.max_iteration, s.conc = int(v[0]), int(v[1]), int(v[2]), int(v[3])
    s.epsilon = float(eps)
    return s


def params_from_record(d: dict) -> CzParams:
    """The parameters as the reference's Build left them (the records that
    oracle/probe/yz_probe_cz.cpp writes; stateio.read_records)."""
    p = CzParams()
    p.nx, p.ny, p.nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    for i in range(4):
        p.bc[i] = int(d["bc"][i])
    for k in ("on_lap", "on_sc", "on_vg", "on_hg", "on_cf", "on_evap", "ev_conc", "ev_spatial", "ev_hast",
              "dt_control", "dt_keep_steps", "c_scheme"):
        setattr(p, k, int(d[k]))
    p.h_lin = _settings(d["h_lin"], d["h_eps"])
    p.c_lin = _settings(d["c_lin"], d["c_eps"])
    for k in ("dx", "dy", "dzeta", "theta_h", "theta_c", "dt", "dt_old", "dt_max", "dt_min", "time",
              "dt_change_factor", "dt_criterion", "dt_scale_floor", "As", "Ma", "Bo", "Pgx", "Pgy", "Sp", "Df", "Ev",
              "coupling_floor"):
        setattr(p, k, float(d[k]))
    p.rot_center[0], p.rot_center[1] = float(d["rot_center"][0]), float(d["rot_center"][1])
    p.visc_c0, p.visc_base, p.visc_exp = (float(x) for x in d["visc"])
    p.sig_c0, p.sig_base, p.sig_coef = (float(x) for x in d["sigma"])
    p.diff_c0, p.diff_base, p.diff_exp = (float(x) for x in d["diff"])
    ev = [float(x) for x in d["evap"]]
    # M_resin, M_solvent, E0, powerN, NegPowExponent, NegPowRmax, ConcR, h_ast, min(dx, dy)
    p.ev_mr, p.ev_ms, p.ev_pown, p.ev_negexp, p.ev_negrmax, p.ev_concr, p.ev_hast_h, p.ev_dr = (
        ev[0], ev[1], ev[3], ev[4], ev[5], ev[6], ev[7], ev[8])
    if ev[2] != 1.0:
        raise ValueError("cz: the evaporation's E0 is taken as 1 (its scale is Ev)")
    return p


def build_pattern(p: CzParams, which: int):
    """(rowptr, col, bc) of the film's (which 0) or the concentration's (1)
    matrix in the reference's storage order; no device needed."""
    L = _bind()
    nnz = _check(L.yz_cz_build_pattern(ctypes.byref(p), which, None, None, None), "yz_cz_build_pattern")
    n = p.nx * p.ny * (p.nz if which else 1)
    rowptr, col, bc = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(n, np.int32)
    _check(L.yz_cz_build_pattern(ctypes.byref(p), which, _ip(rowptr), _ip(col), _ip(bc)), "yz_cz_build_pattern")
    return rowptr, col, bc


class CzModel:
    """One ConcZ model on a CUDA device (yz_cz_*)."""

    def __init__(self, p: CzParams, xc, xf, yc, yf, h, s, c, device: int = 0):
        L = _bind()
        self.p = p
        self.n2, self.n3 = p.nx * p.ny, p.nx * p.ny * p.nz
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (xc, xf, yc, yf, h, s, c)]
        if arr[4].size != self.n2 or arr[5].size != self.n2 or arr[6].size != self.n3:
            raise ValueError("cz: h and s need nx*ny values, c nx*ny*nz")
        self._h = ctypes.c_void_p()
        _check(L.yz_cz_create(device, ctypes.byref(p), *[_fp(a) for a in arr], ctypes.byref(self._h)),
               "yz_cz_create")

    def close(self) -> None:
        if self._h:
            lib().yz_cz_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, nsteps: int) -> dict:
        st = CzStats()
        _check(lib().yz_cz_advance(self._h, int(nsteps), ctypes.byref(st)), "yz_cz_advance")
        return {k: getattr(st, k) for k, _ in CzStats._fields_}

    def fields(self):
        h, c = np.zeros(self.n2), np.zeros(self.n3)
        _check(lib().yz_cz_get_fields(self._h, _fp(h), _fp(c)), "yz_cz_get_fields")
        return h, c

    def fields_into(self, h: np.ndarray, c: np.ndarray) -> None:
        """The fields into caller arrays (pinned host memory, say)."""
        _check(lib().yz_cz_get_fields(self._h, _fp(h), _fp(c)), "yz_cz_get_fields")

    def set_fields(self, h: np.ndarray, c: np.ndarray) -> None:
        _check(lib().yz_cz_set_fields(self._h, _fp(h), _fp(c)), "yz_cz_set_fields")

    def set_precision(self, precision: int) -> None:
        _check(lib().yz_cz_set_precision(self._h, int(precision)), "yz_cz_set_precision")

    def set_amg_reuse(self, max_solves: int) -> None:
        _check(lib().yz_cz_set_amg_reuse(self._h, int(max_solves)), "yz_cz_set_amg_reuse")

    def set_tuning(self, fuse_from: int, coarse_lanes: int, fine_sweeps: int) -> None:
        _check(lib().yz_cz_set_tuning(self._h, int(fuse_from), int(coarse_lanes), int(fine_sweeps)),
               "yz_cz_set_tuning")

    def set_learned(self, cfg=None) -> None:
        """The learned preconditioner of the film's solves
        (yuzen_b200.learned.LearnedConfig, or default_config(); None: off)."""
        from . import learned
        L = learned._bind()
        _check(L.yz_cz_set_learned(self._h, ctypes.byref(cfg) if cfg is not None else None), "yz_cz_set_learned")

    def parts(self) -> dict:
        """The pieces of one step on the present state (yz_cz_parts), by the
        names of oracle/probe/yz_probe_cz.cpp's parts mode."""
        L = lib()
        _check(L.yz_cz_parts(self._h), "yz_cz_parts")
        out = {}
        for name in ("h_A", "h_B", "h_colsrc", "h_qcapx", "h_qexpx", "h_qcapy", "h_qexpy", "h_IA", "h_qx", "h_qy",
                     "h_end", "h_dtdh", "ux", "uy", "c_A", "c_B", "c_rhs", "c_react", "c_qx", "c_qy", "c_w"):
            n = _check(L.yz_cz_read(self._h, name.encode(), None, 0), "yz_cz_read")
            v = np.zeros(n)
            _check(L.yz_cz_read(self._h, name.encode(), _fp(v), n), "yz_cz_read")
            out[name] = v
        return out

    def pattern(self, which: int):
        n = self.n3 if which else self.n2
        nnz = _check(lib().yz_cz_pattern(self._h, which, None, None, None), "yz_cz_pattern")
        rowptr, col, bc = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(n, np.int32)
        _check(lib().yz_cz_pattern(self._h, which, _ip(rowptr), _ip(col), _ip(bc)), "yz_cz_pattern")
        return rowptr, col, bc
