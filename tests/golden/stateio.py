"""Reader of the whole-step probe's output (oracle/probe/yz_probe.cpp) and the
.npz fixtures made from it."""
from __future__ import annotations

from pathlib import Path

import numpy as np

INT_KEYS = (
    "nx", "ny", "bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax",
    "on_laplace", "on_vgrav", "on_pgrav", "on_marangoni", "on_centrifugal", "on_disjoining",
    "on_evap", "conc_field", "slip", "dt_control", "evap_conc_func", "evap_spatial", "evap_hast_modify",
    "nk_max", "nk_min", "jacobi_interval", "lin_precond", "lin_scaling", "lin_maxit", "dt_keep_steps",
    "max_steps", "on_source",
    "conv_height", "conv_conc", "conc_conv", "conc_diff", "lin_c_precond", "lin_c_scaling", "lin_c_maxit",
    "lin_c_conc",
    # the nozzle (SourceBase)
    "src_subregions", "src_supplied",
    # appended after the run
    "steps_done", "diverged",
)
REAL_KEYS = (
    "dx", "dy", "theta", "dt", "dt_max", "dt_min",
    "As", "Ma", "Bo", "Pgx", "Pgy", "Sp", "Dp", "HStar", "Pe", "Mr", "Df", "Ev",
    "L0", "h0", "T0", "lambda", "disj_n", "disj_m", "disj_hstar",
    "visc_c0", "visc_base", "visc_exp", "sig_c0", "sig_base", "sig_coef", "diff_c0", "diff_base", "diff_exp",
    "ev_m_resin", "ev_m_solvent", "ev_e0", "ev_power_n", "ev_negpow_exp", "ev_negpow_rmax", "ev_conc_r", "ev_h_ast",
    "nk_eps", "nk_eps_rel", "lin_eps", "dt_change_factor", "dt_criterion", "dt_scale_floor",
    "x0", "y0", "t_start",
    "xmin", "ymin", "rot_x", "rot_y", "lin_c_eps", "theta_c",
    # the nozzle (SourceBase): radius, flow rate, time constant, arm length and
    # centre, rotation rate, start angle, ramp and plateau times, start time
    "src_radius", "src_rate", "src_tau", "src_arm", "src_arm_x", "src_arm_y", "src_omega", "src_angle0",
    "src_ramp", "src_plateau", "src_t0", "src_conc",
    # appended after the run
    "run_seconds", "t_end",
    # the energy budget (EnergyEval) of the start and the end film
    "energy_F0", "energy_D0", "energy_F1", "energy_D1",
    # with Output.Energy: the energy dissipated over the run, the last step's balance
    "energy_dissipated", "energy_balance",
)
#  BoundaryCondition::tBoundaryCondition (model/BoundaryCondition.h)
BC_NAMES = {0: "Symmetry", 1: "Periodic", 2: "Pinning", 3: "FreshInlet", 4: "Outlet"}


def read_state(path) -> dict:
    raw = Path(path).read_bytes()
    if raw[:8] != b"YZSTATE1":
        raise ValueError(f"{path}: not a probe state")
    off = 8
    ni = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    ints = np.frombuffer(raw, "<i4", ni, off); off += 4 * ni
    nr = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    reals = np.frombuffer(raw, "<f8", nr, off); off += 8 * nr
    if ni != len(INT_KEYS) or nr != len(REAL_KEYS):
        raise ValueError(f"{path}: header has {ni}/{nr} entries, expected {len(INT_KEYS)}/{len(REAL_KEYS)}")
    d = {k: int(v) for k, v in zip(INT_KEYS, ints)}
    d.update({k: float(v) for k, v in zip(REAL_KEYS, reals)})
    m = d["nx"] * d["ny"]
    for k in ("h0", "c0", "s0", "h1", "c1"):
        d["field_" + k] = np.frombuffer(raw, "<f8", m, off).copy(); off += 8 * m
    n = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    nnz = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    d["rowptr"] = np.frombuffer(raw, "<i4", n + 1, off).copy(); off += 4 * (n + 1)
    d["col"] = np.frombuffer(raw, "<i4", nnz, off).copy(); off += 4 * nnz
    d["bc"] = np.frombuffer(raw, "<i4", n, off).copy(); off += 4 * n
    cn = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    cnnz = int(np.frombuffer(raw, "<i4", 1, off)[0]); off += 4
    d["rowptr_c"] = np.frombuffer(raw, "<i4", cn + 1 if cn else 0, off).copy(); off += 4 * (cn + 1 if cn else 0)
    d["col_c"] = np.frombuffer(raw, "<i4", cnnz, off).copy(); off += 4 * cnnz
    return d


def save_npz(path, d: dict) -> None:
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})


def load_npz(path) -> dict:
    z = np.load(path)
    return {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files}


def read_records(path) -> dict:
    """The named records oracle/probe/yz_probe_cz.cpp writes: magic
    "YZCZREC1", then per record the name's length and bytes, its kind (0
    int32, 1 float64), its count and its values.  Single values come back as
    Python scalars, the rest as arrays."""
    raw = Path(path).read_bytes()
    assert raw[:8] == b"YZCZREC1", "not a record file"
    out, o = {}, 8
    while o < len(raw):
        ln = int(np.frombuffer(raw, "<i4", 1, o)[0]); o += 4
        name = raw[o:o + ln].decode(); o += ln
        kind = int(np.frombuffer(raw, "<i4", 1, o)[0]); o += 4
        cnt = int(np.frombuffer(raw, "<i8", 1, o)[0]); o += 8
        dt, sz = ("<i4", 4) if kind == 0 else ("<f8", 8)
        v = np.frombuffer(raw, dt, cnt, o).copy(); o += sz * cnt
        out[name] = (int(v[0]) if kind == 0 else float(v[0])) if cnt == 1 and name not in ARRAY_RECORDS else v
    return out


#  records that stay arrays even when they hold one value
ARRAY_RECORDS = {"rot_center", "bc", "h_lin", "c_lin", "visc", "sigma", "diff", "evap"}
