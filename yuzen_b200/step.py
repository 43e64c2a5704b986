"""ctypes binding of the whole-step seam of include/yuzen_b200.h (yz_step_*):
the implicit time step of the well-mixed film-height equation on the device,
C_NewtonKantorovich::TimeAdvance (NewtonKantorovich.cpp:424-486) with the
hooks of WellMixed_HeightEquationBase, in the reference's non-dimensional
variables."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _Settings, _check, _fp, _ip, lib

_f64p = ctypes.POINTER(ctypes.c_double)


class StepParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("bc", ctypes.c_int * 4),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("xmin", ctypes.c_double), ("ymin", ctypes.c_double),
        ("theta", ctypes.c_double),
        ("on_laplace", ctypes.c_int), ("on_vgrav", ctypes.c_int), ("on_pgrav", ctypes.c_int),
        ("on_marangoni", ctypes.c_int), ("on_centrifugal", ctypes.c_int), ("on_disjoining", ctypes.c_int),
        ("on_evap", ctypes.c_int), ("conc_field", ctypes.c_int),
        ("Bo", ctypes.c_double), ("Dp", ctypes.c_double), ("hstar", ctypes.c_double), ("disj_n", ctypes.c_double),
        ("disj_m", ctypes.c_double), ("lambda_slip", ctypes.c_double), ("Ev", ctypes.c_double),
        ("visc_c0", ctypes.c_double), ("visc_base", ctypes.c_double), ("visc_exp", ctypes.c_double),
        ("sig_c0", ctypes.c_double), ("sig_base", ctypes.c_double), ("sig_coef", ctypes.c_double),
        ("ev_conc_func", ctypes.c_int), ("ev_spatial", ctypes.c_int), ("ev_hast_modify", ctypes.c_int),
        ("ev_m_resin", ctypes.c_double), ("ev_m_solvent", ctypes.c_double), ("ev_power_n", ctypes.c_double),
        ("ev_conc_r", ctypes.c_double), ("ev_negpow_exp", ctypes.c_double), ("ev_negpow_rmax", ctypes.c_double),
        ("ev_h_ast", ctypes.c_double),
        ("nk_max", ctypes.c_int), ("nk_min", ctypes.c_int), ("nk_eps", ctypes.c_double), ("nk_eps_rel", ctypes.c_double),
        ("lin", _Settings),
        ("dt_control", ctypes.c_int), ("dt_keep_steps", ctypes.c_int),
        ("dt", ctypes.c_double), ("dt_max", ctypes.c_double), ("dt_min", ctypes.c_double),
        ("dt_change_factor", ctypes.c_double), ("dt_criterion", ctypes.c_double), ("dt_scale_floor", ctypes.c_double),
        ("t_start", ctypes.c_double),
        ("conv_height", ctypes.c_int),
        ("Pgx", ctypes.c_double), ("Pgy", ctypes.c_double),
        ("Sp", ctypes.c_double), ("rot_x", ctypes.c_double), ("rot_y", ctypes.c_double),
        ("As", ctypes.c_double), ("Ma", ctypes.c_double),
        ("conv_conc", ctypes.c_int), ("conc_convection", ctypes.c_int), ("conc_diffusion", ctypes.c_int),
        ("theta_c", ctypes.c_double),
        ("Df", ctypes.c_double), ("diff_c0", ctypes.c_double), ("diff_base", ctypes.c_double),
        ("diff_exp", ctypes.c_double),
        ("lin_conc", _Settings),
        ("on_source", ctypes.c_int), ("src_subregions", ctypes.c_int),
        ("src_radius", ctypes.c_double), ("src_rate", ctypes.c_double), ("src_tau", ctypes.c_double),
        ("src_arm", ctypes.c_double), ("src_arm_x", ctypes.c_double), ("src_arm_y", ctypes.c_double),
        ("src_omega", ctypes.c_double), ("src_angle0", ctypes.c_double), ("src_ramp", ctypes.c_double),
        ("src_plateau", ctypes.c_double), ("src_t0", ctypes.c_double),
        ("src_supplied", ctypes.c_int), ("src_conc", ctypes.c_double),
    ]


class StepStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int), ("newton_iterations", ctypes.c_int), ("linear_iterations", ctypes.c_int),
        ("retries", ctypes.c_int), ("time", ctypes.c_double), ("dt", ctypes.c_double),
        ("last_resid", ctypes.c_double), ("setup_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("assemble_ms", ctypes.c_double), ("device_ms", ctypes.c_double), ("launches", ctypes.c_longlong),
        ("conc_iterations", ctypes.c_int), ("conc_solves", ctypes.c_int),
        ("energy_F", ctypes.c_double), ("energy_D", ctypes.c_double),
        ("energy_dissipated", ctypes.c_double), ("energy_balance", ctypes.c_double),
        ("amg_setups", ctypes.c_int),
        ("learned_solves", ctypes.c_int), ("learned_fallbacks", ctypes.c_int), ("learned_iterations", ctypes.c_int),
        ("learned_samples", ctypes.c_int), ("learned_train_ms", ctypes.c_double), ("learned_val_err", ctypes.c_double),
        ("learned_loss", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def params_from_state(d: dict) -> StepParams:
    """The step parameters of a case as the reference's model holds them
    (the dict of the whole-step probe, tests/golden/stateio.py, or of
    yuzen_b200.cases)."""
    p = StepParams()
    p.nx, p.ny = d["nx"], d["ny"]
    for e, k in enumerate(("bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax")):
        p.bc[e] = d[k]
    p.dx, p.dy, p.xmin, p.ymin, p.theta = d["dx"], d["dy"], d["xmin"], d["ymin"], d["theta"]
    p.on_laplace, p.on_vgrav, p.on_pgrav = d["on_laplace"], d["on_vgrav"], d["on_pgrav"]
    p.on_marangoni, p.on_centrifugal, p.on_disjoining = d["on_marangoni"], d["on_centrifugal"], d["on_disjoining"]
    p.on_evap, p.conc_field = d["on_evap"], d["conc_field"]
    p.Bo, p.Dp, p.hstar = d["Bo"], d["Dp"], d["disj_hstar"]
    p.disj_n, p.disj_m, p.lambda_slip, p.Ev = d["disj_n"], d["disj_m"], d["lambda"], d["Ev"]
    p.visc_c0, p.visc_base, p.visc_exp = d["visc_c0"], d["visc_base"], d["visc_exp"]
    p.sig_c0, p.sig_base, p.sig_coef = d["sig_c0"], d["sig_base"], d["sig_coef"]
    p.ev_conc_func, p.ev_spatial, p.ev_hast_modify = d["evap_conc_func"], d["evap_spatial"], d["evap_hast_modify"]
    p.ev_m_resin, p.ev_m_solvent, p.ev_power_n = d["ev_m_resin"], d["ev_m_solvent"], d["ev_power_n"]
    p.ev_conc_r, p.ev_negpow_exp, p.ev_negpow_rmax = d["ev_conc_r"], d["ev_negpow_exp"], d["ev_negpow_rmax"]
    p.ev_h_ast = d["ev_h_ast"]
    p.nk_max, p.nk_min, p.nk_eps, p.nk_eps_rel = d["nk_max"], d["nk_min"], d["nk_eps"], d["nk_eps_rel"]
    p.lin = _Settings(d["lin_precond"], d["lin_scaling"], d["lin_maxit"], d["lin_eps"], 0)
    p.dt_control, p.dt_keep_steps = d["dt_control"], d["dt_keep_steps"]
    p.dt, p.dt_max, p.dt_min = d["dt"], d["dt_max"], d["dt_min"]
    p.dt_change_factor, p.dt_criterion, p.dt_scale_floor = d["dt_change_factor"], d["dt_criterion"], d["dt_scale_floor"]
    p.t_start = d["t_start"]
    p.conv_height = d["conv_height"]
    p.Pgx, p.Pgy, p.Sp, p.rot_x, p.rot_y = d["Pgx"], d["Pgy"], d["Sp"], d["rot_x"], d["rot_y"]
    p.As, p.Ma = d["As"], d["Ma"]
    p.conv_conc, p.conc_convection, p.conc_diffusion = d["conv_conc"], d["conc_conv"], d["conc_diff"]
    p.theta_c = d["theta_c"]
    p.Df, p.diff_c0, p.diff_base, p.diff_exp = d["Df"], d["diff_c0"], d["diff_base"], d["diff_exp"]
    p.lin_conc = _Settings(d["lin_c_precond"], d["lin_c_scaling"], d["lin_c_maxit"], d["lin_c_eps"], d["lin_c_conc"])
    # the nozzle (fixtures written before the probe dumped it have none)
    p.on_source = int(d.get("on_source", 0))
    p.src_subregions = int(d.get("src_subregions", 1))
    for k in ("radius", "rate", "tau", "arm", "arm_x", "arm_y", "omega", "angle0", "ramp", "plateau", "t0"):
        setattr(p, "src_" + k, float(d.get("src_" + k, 0.0)))
    p.src_supplied = int(d.get("src_supplied", 0))
    p.src_conc = float(d.get("src_conc", 0.0))
    return p


_BOUND = False


def _bind():
    global _BOUND
    if _BOUND:
        return lib()
    L = lib()
    L.yz_step_create.argtypes = [ctypes.c_int, ctypes.POINTER(StepParams), _f64p, _f64p, _f64p,
                                 ctypes.POINTER(ctypes.c_void_p)]
    L.yz_step_destroy.argtypes = [ctypes.c_void_p]
    L.yz_step_advance.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StepStats)]
    L.yz_step_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_step_set_amg_reuse.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_step_set_graph_loop.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_step_set_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.yz_step_energy.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_step_set_energy.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.yz_step_get_fields.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_step_set_fields.argtypes = [ctypes.c_void_p, _f64p, _f64p]
    L.yz_launch_count.restype = ctypes.c_longlong
    L.yz_step_pattern.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)]
    L.yz_step_system.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_double, _f64p, _f64p]
    L.yz_step_conc_pattern.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.yz_step_conc_system.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_double, _f64p, _f64p]
    L.yz_pattern_2d.argtypes = [ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    _BOUND = True
    return L


class Step:
    """The device step of one case: Step(params, h, c, s); advance(n)."""

    def __init__(self, params: StepParams, h, c, s, device: int = 0):
        L = _bind()
        self.params = params
        self.n = params.nx * params.ny
        h, c, s = (np.ascontiguousarray(a, np.float64) for a in (h, c, s))
        if not (h.size == c.size == s.size == self.n):
            raise ValueError("h, c and s need nx*ny values each")
        self._h = ctypes.c_void_p()
        _check(L.yz_step_create(device, ctypes.byref(params), _fp(h), _fp(c), _fp(s), ctypes.byref(self._h)),
               "yz_step_create")

    def set_precision(self, precision: int) -> None:
        """The preconditioner arithmetic of the step's solves (PREC_FP64, or
        PREC_FP32_CYCLE: the V-cycle in float inside the FP64 BiCGStab)."""
        _check(lib().yz_step_set_precision(self._h, precision), "yz_step_set_precision")

    def set_amg_reuse(self, max_solves: int) -> None:
        """AMG hierarchy reuse of the step's solves (0: a new set-up every
        solve, the reference's way; k > 0: a set-up serves up to k further
        solves)."""
        _check(lib().yz_step_set_amg_reuse(self._h, max_solves), "yz_step_set_amg_reuse")

    def set_graph_loop(self, on: bool) -> None:
        """The step's BiCGStab loops as CUDA graph launches (default) or
        from the stream (yz_step_set_graph_loop)."""
        _check(lib().yz_step_set_graph_loop(self._h, int(bool(on))), "yz_step_set_graph_loop")

    def set_tuning(self, fuse_from: int = -1, coarse_lanes: int = 0, fine_sweeps: int = 0) -> None:
        """The FP32 V-cycle's shape (yz_step_set_tuning): the first fused level
        (-1 default, 0 none), the coarse levels' lanes a row (0: by row
        length) and the finest level's post-smoothing sweeps (0: default)."""
        _check(lib().yz_step_set_tuning(self._h, int(fuse_from), int(coarse_lanes), int(fine_sweeps)),
               "yz_step_set_tuning")

    def set_learned(self, cfg=None) -> None:
        """The learned preconditioner of the film's solves
        (yuzen_b200.learned.LearnedConfig, or default_config(); None: off)."""
        from . import learned
        L = learned._bind()
        _check(L.yz_step_set_learned(self._h, ctypes.byref(cfg) if cfg is not None else None), "yz_step_set_learned")

    def state(self) -> np.ndarray:
        """The state a later step depends on (yz_step_get_state), a float64
        array that set_state takes back."""
        L = lib()
        L.yz_step_state_size.restype = ctypes.c_longlong
        L.yz_step_state_size.argtypes = [ctypes.c_void_p]
        out = np.zeros(int(L.yz_step_state_size(self._h)))
        _check(L.yz_step_get_state(self._h, _fp(out)), "yz_step_get_state")
        return out

    def set_state(self, state: np.ndarray) -> None:
        """Continue from a state taken with state() (yz_step_set_state)."""
        L = lib()
        L.yz_step_set_state.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_longlong]
        a = np.ascontiguousarray(state, np.float64)
        _check(L.yz_step_set_state(self._h, _fp(a), a.size), "yz_step_set_state")

    def write_field(self, path, case) -> None:
        """The film as a field file in the reference's ASCII format (columns
        x y h+s u v c h s over grid points 1..nx-2 x 1..ny-2, non-dimensional;
        Output.cpp:902-912), which its restart reads back (Restart.h:36-42):
        `case` is the yuzen_b200.cases.Case the step was built from."""
        h, c = self.fields()
        case.write_fields(path, h, c)

    def energy(self):
        """(F, D): the free energy of the film the step holds and the flux
        power of the potential (the reference's EnergyEval)."""
        F, D = ctypes.c_double(), ctypes.c_double()
        _check(lib().yz_step_energy(self._h, ctypes.byref(F), ctypes.byref(D)), "yz_step_energy")
        return F.value, D.value

    def set_energy(self, on: bool) -> None:
        """The energy history (Output.Energy): the budget of the present film,
        then every step's, with the energy dissipated and the last step's
        balance in advance()'s stats (yz_step_set_energy)."""
        _check(lib().yz_step_set_energy(self._h, int(bool(on))), "yz_step_set_energy")

    def advance(self, nsteps: int = 1) -> dict:
        st = StepStats()
        _check(lib().yz_step_advance(self._h, nsteps, ctypes.byref(st)), "yz_step_advance")
        return st.as_dict()

    def fields(self):
        h = np.zeros(self.n)
        c = np.zeros(self.n)
        _check(lib().yz_step_get_fields(self._h, _fp(h), _fp(c)), "yz_step_get_fields")
        return h, c

    def fields_into(self, h: np.ndarray, c: np.ndarray | None = None) -> None:
        """Download the fields into caller-owned (e.g. pinned) float64 arrays."""
        _check(lib().yz_step_get_fields(self._h, _fp(h), _fp(c) if c is not None else None), "yz_step_get_fields")

    def set_fields(self, h: np.ndarray, c: np.ndarray | None = None) -> None:
        """Upload the fields the next step starts from (host arrays)."""
        _check(lib().yz_step_set_fields(self._h, _fp(h), _fp(c) if c is not None else None), "yz_step_set_fields")

    def pattern(self):
        L = lib()
        nnz = _check(L.yz_step_pattern(self._h, None, None, None), "yz_step_pattern")
        rowptr = np.zeros(self.n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        bc = np.zeros(self.n, np.int32)
        _check(L.yz_step_pattern(self._h, _ip(rowptr), _ip(col), _ip(bc)), "yz_step_pattern")
        return rowptr, col, bc

    def system(self, h_old, h, dt: float):
        h_old = np.ascontiguousarray(h_old, np.float64)
        h = np.ascontiguousarray(h, np.float64)
        rowptr, col, bc = self.pattern()
        ia = np.zeros(col.size)
        rhs = np.zeros(self.n)
        _check(lib().yz_step_system(self._h, _fp(h_old), _fp(h), float(dt), _fp(ia), _fp(rhs)), "yz_step_system")
        return ia, rhs

    def conc_pattern(self):
        """The concentration equation's CRS pattern (rowptr, col); empty
        arrays without the concentration equation."""
        L = lib()
        nnz = _check(L.yz_step_conc_pattern(self._h, None, None), "yz_step_conc_pattern")
        if nnz == 0:
            return np.zeros(0, np.int32), np.zeros(0, np.int32)
        rowptr = np.zeros(self.n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        _check(L.yz_step_conc_pattern(self._h, _ip(rowptr), _ip(col)), "yz_step_conc_pattern")
        return rowptr, col

    def conc_system(self, h, c, dt: float):
        """The first Newton pass's concentration system of a step from the
        committed (h, c): (values in storage order, right-hand side)."""
        h = np.ascontiguousarray(h, np.float64)
        c = np.ascontiguousarray(c, np.float64)
        rowptr, col = self.conc_pattern()
        val = np.zeros(col.size)
        rhs = np.zeros(self.n)
        _check(lib().yz_step_conc_system(self._h, _fp(h), _fp(c), float(dt), _fp(val), _fp(rhs)),
               "yz_step_conc_system")
        return val, rhs

    def close(self) -> None:
        if self._h:
            lib().yz_step_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pattern_2d(params: StepParams):
    """The CRS pattern of the step, built on the host (no device needed):
    (rowptr, col, bc)."""
    L = _bind()
    nnz = _check(L.yz_pattern_2d(ctypes.byref(params), None, None, None), "yz_pattern_2d")
    n = params.nx * params.ny
    rowptr = np.zeros(n + 1, np.int32)
    col = np.zeros(nnz, np.int32)
    bc = np.zeros(n, np.int32)
    _check(L.yz_pattern_2d(ctypes.byref(params), _ip(rowptr), _ip(col), _ip(bc)), "yz_pattern_2d")
    return rowptr, col, bc


def launch_count() -> int:
    """Kernels the library launched in this process."""
    return int(_bind().yz_launch_count())
