"""Seeded synthetic cases of the implicit step, in the reference's own case
format (TOML + an ASCII field restart) and as the non-dimensional state the
device step starts from.

The reference builds its non-dimensional state in
NonDimensionalNumbers::Build (model/NonDimensionalNumbers.cpp:43-140), the
grid in C_Grid2D::Build / RectGrid::SetExtentX (model/Grids.cpp:95-109,
grid/RectGrid.h:459-465), the time-step limits in WellMixed_ModelBase::Build
and ::Run (WellMixedModelBase.h:440-467, 1235-1250), and reads a seeded
initial film through C_Restart::ReadAscii_WM2D (IO/Restart.cpp:280-316),
after which BoundaryCondition2D::ApplyToField makes every ghost an exact copy
of its partner (BoundaryCondition.cpp:309-372).  This module restates those
steps with the same floating-point operations (Python floats are IEEE
doubles, math.pow/sqrt/atan are the C library's), so the state it hands the
device is the reference's own to the bit; tests/test_cases.py checks that
against the whole-step probe.

    cfg = spinodal_224()              # the 224^2 spinodal film
    state = cfg.state()               # dict: params + fields (nx*ny each)
    cfg.write_reference(workdir)      # case.toml + init.dat for the reference
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

GG = 9.80665
PI = 4.0 * math.atan(1.0)   # Math::pi(), MyMath.h:110

#  BoundaryCondition::tBoundaryCondition
BC = {"Symmetry": 0, "Periodic": 1, "Pinning": 2, "FreshInlet": 3, "Outlet": 4}
#  C_Interpolation_base4::t_Scheme by its Numerics.Convection key (FiniteDifferences.cpp:216-226)
SCHEMES = {"Upwind1": 0, "Upwind2": 1, "Central2": 2, "UTOPIA": 3, "QUICK": 4, "KK": 5, "Central4": 6,
           "Koren": 7, "VanLeer": 8}


def _toml_value(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return repr(v)
    if isinstance(v, str):
        return '"' + v + '"'
    if isinstance(v, (list, tuple)):
        return "[" + ", ".join(_toml_value(x) for x in v) + "]"
    raise TypeError(type(v))


def toml_dumps(doc: dict) -> str:
    out: list[str] = []

    def emit(t: dict, prefix: str) -> None:
        sc = [(k, v) for k, v in t.items() if not isinstance(v, dict)]
        sub = [(k, v) for k, v in t.items() if isinstance(v, dict)]
        if prefix:
            out.append(f"[{prefix}]")
        out.extend(f"{k} = {_toml_value(v)}" for k, v in sc)
        out.append("")
        for k, v in sub:
            emit(v, f"{prefix}.{k}" if prefix else k)

    emit(doc, "")
    return "\n".join(out) + "\n"


@dataclass
class Case:
    """A well-mixed 2-D case: fluid, physics switches, grid, numerics and a
    seeded initial film (interior cells, non-dimensional)."""
    name: str
    Nx: int
    Ny: int
    xlim: tuple            # dimensional [m]
    ylim: tuple
    h0: float              # TotalHeight [m]
    precursor: float       # PrecursorRatio
    bc: tuple              # Xmin, Xmax, Ymin, Ymax names
    dt: float              # InitialDt [s]
    steps: int = 12
    end_time: float = 1e30
    dt_control: bool = False
    fluid: dict = field(default_factory=lambda: {
        "rho": 1000.0, "sigma": 30.0e-3, "sigma_c0": 0.5, "sigma_coef": 10e-3,
        "mu": 100.0e-3, "mu_c0": 0.5, "mu_exp": 10.0, "D": 1.0e-9, "D_c0": 0.5, "D_exp": -7.0,
        "M_solvent": 100.0, "M_resin": 2000.0})
    length_scale: float | None = None   # custom L0 [m], else the capillary length
    laplace: bool = True
    vgrav: float | None = None          # Acceleration [m/s^2], None: off
    hgrav: tuple | None = None          # [gx, gy]
    centrifugal: tuple | None = None    # (omega [rad/s], [x, y] axis)
    marangoni: bool = False
    disjoining: tuple | None = None     # (theta_e [deg], n, m)
    evaporation: dict | None = None     # {"Coef":..., "ConcFunc":..., "SpatialFunc":...}
    slip: float | None = None           # slip length [m]
    conc_model: str = "None"            # "None" | "WM"
    conc0: float = 0.5
    h_init: np.ndarray | None = None    # (Ny, Nx) interior film, non-dimensional
    s_init: np.ndarray | None = None
    c_init: np.ndarray | None = None
    conv_height: str = "Koren"          # Numerics.Convection.Height
    conv_conc: str = "UTOPIA"           # Numerics.Convection.Concentration
    newton: dict = field(default_factory=lambda: {"max": 50, "min": 1, "eps": 1e-12, "eps_rel": 1e-6})
    linear: dict = field(default_factory=lambda: {"maxit": 8000, "eps": 1e-13, "precond": "ILU", "scaling": True})
    dtc: dict = field(default_factory=lambda: {"MaxDtFactor": 1.0e10, "MinDt": 1.0e-15, "Criterion": 1e-3,
                                               "KeepSteps": 50, "ChangeFactor": 0.75, "ScaleFloor": 0.0})

    # ------------------------------------------------------------------
    def toml(self, restart_file: str = "init.dat") -> dict:
        f = self.fluid
        doc = {
            "SolverName": "Yuzen-1.0", "InputFormatVersion": "1.0", "JobName": self.name,
            "Grid": {"Dimension": "xyh", "Xmin": self.xlim[0], "Xmax": self.xlim[1], "Ymin": self.ylim[0],
                     "Ymax": self.ylim[1], "Nx": self.Nx, "Ny": self.Ny, "Nz": 1},
            "Initial": {"Concentration": {"Type": "uniform", "Value": self.conc0},
                        "SurfaceShape": {"TotalHeight": self.h0, "PrecursorRatio": self.precursor}},
            "Substrate": {"TotalHeight": 0.0},
            "Fluid": {"Name": "synthetic", "Density": {"Value": f["rho"]},
                      "SurfaceTension": {"BaseValue": f["sigma"], "BaseConc": f["sigma_c0"], "Coef": f["sigma_coef"]},
                      "Viscosity": {"BaseValue": f["mu"], "BaseConc": f["mu_c0"], "Exponent": f["mu_exp"]},
                      "Diffusivity": {"BaseValue": f["D"], "BaseConc": f["D_c0"], "Exponent": f["D_exp"]},
                      "MolarMass": {"Solvent": f["M_solvent"], "Resin": f["M_resin"]}},
            "Physics": {
                "ConcField": {"Model": self.conc_model, "EnableConvection": True, "EnableDiffusion": True},
                "LaplacePressure": {"Enable": self.laplace},
                "SolutoCapillarity": {"Enable": self.marangoni},
                "VerticalGravity": {"Enable": self.vgrav is not None,
                                    "Acceleration": self.vgrav if self.vgrav is not None else 9.80665},
                "HorizontalGravity": {"Enable": self.hgrav is not None,
                                      "Acceleration": list(self.hgrav) if self.hgrav else [0.0, 0.0]},
                "Centrifugal": {"Enable": self.centrifugal is not None,
                                "RotationRate": self.centrifugal[0] if self.centrifugal else 0.0,
                                "RotationAxis": list(self.centrifugal[1]) if self.centrifugal else [0.0, 0.0]},
                "Evaporation": {"Enable": self.evaporation is not None,
                                **({"Coef": 1e-7, "ConcFunc": "Raoult", "SpatialFunc": "uniform",
                                    "NegPowExponent": 0.25, "NegPowRmax": 75e-3} | (self.evaporation or {}))},
                "DisjoiningPressure": {"Enable": self.disjoining is not None,
                                       "ContactAngle": self.disjoining[0] if self.disjoining else 10.0,
                                       "ExponentN": self.disjoining[1] if self.disjoining else 3.0,
                                       "ExponentM": self.disjoining[2] if self.disjoining else 2.0},
                "Slip": {"Enable": self.slip is not None, "Length": self.slip if self.slip else 0.0},
                "Source": {"Enable": False},
            },
            "Boundary": {"XminBC": {"Type": self.bc[0]}, "XmaxBC": {"Type": self.bc[1]},
                         "YminBC": {"Type": self.bc[2]}, "YmaxBC": {"Type": self.bc[3]}},
            "Output": {"Dimensioned": False, "Overwrite": True,
                       "FieldData": {"TimeInterval": 1e30, "NeutralFile": False, "VTKFile": False},
                       "GeneralHistory": {"TimeInterval": 1e30}, "CalcInfo": {"TimeInterval": 1e30},
                       "ProbeList": {"TimeInterval": 1e30}},
            "Numerics": {
                "InitialDt": self.dt, "MaxSteps": self.steps, "EndTime": self.end_time,
                "Convection": {"Height": self.conv_height, "Concentration": self.conv_conc},
                "TimeStepControl": {"Enable": self.dt_control, **self.dtc},
                "HeightEquation": {"NewtonMaxIterations": self.newton["max"],
                                   "NewtonMinIterations": self.newton["min"],
                                   "NewtonEpsilon": self.newton["eps"], "NewtonEpsilonRel": self.newton["eps_rel"],
                                   "LinearSolver": {"Backend": "amgcl", "MaxIterations": self.linear["maxit"],
                                                    "Epsilon": self.linear["eps"], "RowScaling": self.linear["scaling"],
                                                    "PreconditionType": self.linear["precond"]}},
                "ConcEquation": {"LinearSolver": {"Backend": "amgcl", "MaxIterations": 5000, "Epsilon": 1e-13,
                                                  "RowScaling": True, "PreconditionType": "ILU"}},
            },
            "Restart": {"Enable": True, "ASCII": True, "FileName": restart_file, "RestartTime": 0.0, "FileIndex": 0},
        }
        if self.length_scale is not None:
            doc["LengthScaleType"] = "custom"
            doc["LengthScale"] = self.length_scale
        return doc

    # ------------------------------------------------------------------
    def scales(self) -> dict:
        """NonDimensionalNumbers::Build (NonDimensionalNumbers.cpp:43-140)."""
        f = self.fluid
        sig0, rho = f["sigma"], f["rho"]
        L0 = math.sqrt(sig0 / (rho * GG))
        if self.length_scale is not None:
            L0 = self.length_scale
        h0 = self.h0
        eps = h0 / L0
        mu0, sigC = f["mu"], f["sigma_coef"]
        Gz = self.vgrav if self.vgrav is not None else 9.80665
        Gx, Gy = self.hgrav if self.hgrav else (0.0, 0.0)
        omega = self.centrifugal[0] if self.centrifugal else 0.0
        D0 = f["D"]
        E0 = (self.evaporation or {}).get("Coef", 1e-7)
        T0 = mu0 * math.pow(L0, 4.0) / (sig0 * math.pow(h0, 3.0))
        s = {"L0": L0, "h0": h0, "T0": T0, "U0": L0 / T0}
        s["As"] = math.pow(eps, -2.0)
        s["Ma"] = sigC / sig0
        s["Bo"] = rho * Gz * math.pow(L0, 2.0) / sig0
        s["Pgx"] = rho * Gx * math.pow(L0, 2.0) / sig0 / eps
        s["Pgy"] = rho * Gy * math.pow(L0, 2.0) / sig0 / eps
        s["Sp"] = rho * math.pow(omega, 2.0) * math.pow(L0, 4.0) / (sig0 * h0)
        s["HStar"] = self.precursor
        s["Dp"] = 0.0
        if self.disjoining is not None:
            th_deg, nn, mm = self.disjoining
            th = th_deg * PI / 180.0
            s["Dp"] = s["As"] * (nn - 1.0) * (mm - 1.0) / (2.0 * s["HStar"] * (nn - mm)) * th * th
        s["Pe"] = E0 * h0 / D0
        s["Mr"] = f["M_resin"] / f["M_solvent"]
        s["Ev"] = E0 * T0 / h0
        s["Df"] = D0 * T0 / math.pow(L0, 2.0)
        if self.vgrav is None:
            s["Bo"] = 0.0
        if self.hgrav is None:
            s["Pgx"] = s["Pgy"] = 0.0
        if self.centrifugal is None:
            s["Sp"] = 0.0
        if not self.marangoni:
            s["Ma"] = 0.0
        s["lambda"] = self.slip / h0 if self.slip else 0.0
        return s

    def grid(self, L0: float) -> dict:
        """C_Grid2D::Build + RectGrid::SetExtentX on the non-dimensional extent."""
        out = {}
        for ax, lim, N in (("x", self.xlim, self.Nx), ("y", self.ylim, self.Ny)):
            lo, hi = lim[0] / L0, lim[1] / L0
            d0 = (hi - lo) / float(N)
            gmin, gmax = lo - 2 * d0, hi + 2 * d0
            n = N + 4
            d = (gmax - gmin) / n
            out["d" + ax] = d
            out[ax + "min"] = gmin
            out[ax + "0"] = gmin + 0 * d + d * 0.5
            out["n" + ax] = n
        return out

    # ------------------------------------------------------------------
    def fields(self):
        """h, c, s on the whole grid (nx*ny, row iy*nx + ix), ghosts copied
        from their partners as BoundaryCondition2D::ApplyToField leaves them."""
        nx, ny = self.Nx + 4, self.Ny + 4
        H = np.zeros((ny, nx))
        S = np.zeros((ny, nx))
        C = np.full((ny, nx), float(self.conc0))
        H[2:-2, 2:-2] = self.h_init
        if self.s_init is not None:
            S[2:-2, 2:-2] = self.s_init
        if self.c_init is not None:
            C[2:-2, 2:-2] = self.c_init
        bx = [BC[self.bc[0]], BC[self.bc[1]]]
        by = [BC[self.bc[2]], BC[self.bc[3]]]

        def partner(a, n, lo, hi):
            if a < 2:
                return a + (n - 4) if lo == 1 else 3 - a
            if a >= n - 2:
                return a - (n - 4) if hi == 1 else 2 * (n - 2) - 1 - a
            return a

        px = np.array([partner(a, nx, *bx) for a in range(nx)])
        py = np.array([partner(a, ny, *by) for a in range(ny)])
        for A in (H, S, C):
            A[:, :] = A[np.ix_(py, px)]
        return H.ravel(), C.ravel(), S.ravel()

    def state(self) -> dict:
        """The non-dimensional state of the step (the keys of the whole-step
        probe, tests/golden/stateio.py)."""
        sc = self.scales()
        g = self.grid(sc["L0"])
        ev = self.evaporation or {}
        f = self.fluid
        dt = self.dt / sc["T0"]
        dxmin = min(g["dx"], g["dy"])
        dt_max = self.dtc["MaxDtFactor"] * math.pow(dxmin, 4.0)
        cap = 1e30 / sc["T0"]
        if cap < dt_max:
            dt_max = cap
        if dt_max < dt:
            dt = dt_max
        h, c, s = self.fields()
        return {
            "nx": g["nx"], "ny": g["ny"], "bc_xmin": BC[self.bc[0]], "bc_xmax": BC[self.bc[1]],
            "bc_ymin": BC[self.bc[2]], "bc_ymax": BC[self.bc[3]],
            "on_laplace": int(self.laplace), "on_vgrav": int(self.vgrav is not None),
            "on_pgrav": int(self.hgrav is not None), "on_marangoni": int(self.marangoni),
            "on_centrifugal": int(self.centrifugal is not None), "on_disjoining": int(self.disjoining is not None),
            "on_evap": int(self.evaporation is not None), "conc_field": int(self.conc_model == "WM"),
            "slip": int(bool(self.slip)), "dt_control": int(self.dt_control),
            "evap_conc_func": 1 if ev.get("ConcFunc") == "PowerN" else 0,
            "evap_spatial": 1 if ev.get("SpatialFunc") == "negPow" else 0,
            "nk_max": self.newton["max"], "nk_min": self.newton["min"], "jacobi_interval": 1,
            "lin_precond": {"None": 0, "Jacobi": 1, "ILU": 2}[self.linear["precond"]],
            "lin_scaling": int(self.linear["scaling"]), "lin_maxit": self.linear["maxit"],
            "dt_keep_steps": self.dtc["KeepSteps"], "max_steps": self.steps, "on_source": 0,
            "dx": g["dx"], "dy": g["dy"], "theta": 0.5, "dt": dt, "dt_max": dt_max, "dt_min": self.dtc["MinDt"],
            "As": sc["As"], "Ma": sc["Ma"], "Bo": sc["Bo"], "Pgx": sc["Pgx"], "Pgy": sc["Pgy"], "Sp": sc["Sp"],
            "Dp": sc["Dp"], "HStar": sc["HStar"], "Pe": sc["Pe"], "Mr": sc["Mr"], "Df": sc["Df"], "Ev": sc["Ev"],
            "L0": sc["L0"], "h0": sc["h0"], "T0": sc["T0"], "lambda": sc["lambda"],
            "disj_n": self.disjoining[1] if self.disjoining else 3.0,
            "disj_m": self.disjoining[2] if self.disjoining else 2.0, "disj_hstar": sc["HStar"],
            "visc_c0": f["mu_c0"], "visc_base": 1.0, "visc_exp": f["mu_exp"],
            "sig_c0": f["sigma_c0"], "sig_base": 1.0, "sig_coef": sc["Ma"],
            "diff_c0": f["D_c0"], "diff_base": 1.0, "diff_exp": f["D_exp"],
            **self._evap_params(sc),
            "nk_eps": self.newton["eps"], "nk_eps_rel": self.newton["eps_rel"], "lin_eps": self.linear["eps"],
            "dt_change_factor": self.dtc["ChangeFactor"], "dt_criterion": self.dtc["Criterion"],
            "dt_scale_floor": self.dtc["ScaleFloor"], "x0": g["x0"], "y0": g["y0"], "t_start": 0.0,
            "xmin": g["xmin"], "ymin": g["ymin"],
            "rot_x": (self.centrifugal[1][0] if self.centrifugal else 0.0) / sc["L0"],
            "rot_y": (self.centrifugal[1][1] if self.centrifugal else 0.0) / sc["L0"],
            "conv_height": SCHEMES[self.conv_height], "conv_conc": SCHEMES[self.conv_conc],
            "conc_conv": 1, "conc_diff": 1,
            **self._conc_solver(),
            "field_h0": h, "field_c0": c, "field_s0": s,
        }

    def _conc_solver(self) -> dict:
        """The concentration equation's linear solver as the model holds it:
        Numerics.ConcEquation.LinearSolver with the concentration role when
        ConcField = WM; the LinearSolver defaults otherwise (the equation is
        not built, LinearSolverBackend.h:48-50)."""
        if self.conc_model == "WM":
            return {"lin_c_precond": 2, "lin_c_scaling": 1, "lin_c_maxit": 5000, "lin_c_eps": 1e-13,
                    "lin_c_conc": 1, "theta_c": 0.5}
        return {"lin_c_precond": 2, "lin_c_scaling": 1, "lin_c_maxit": 100, "lin_c_eps": 1e-12,
                "lin_c_conc": 0, "theta_c": 0.5}

    def _evap_params(self, sc: dict) -> dict:
        """C_Evaporation as NonDimensionalNumbers builds it (Coef 1, resin
        molar mass Mr, solvent 1); left at its constructor's values when the
        term is off (Evaporation.cpp:20-34)."""
        ev = self.evaporation
        if ev is None:
            return {"ev_m_resin": 1.0, "ev_m_solvent": 1.0, "ev_e0": 1.0, "ev_power_n": 1.0,
                    "ev_negpow_exp": 0.25, "ev_negpow_rmax": 1.0, "ev_conc_r": 0.0, "ev_h_ast": 0.0,
                    "evap_hast_modify": 0}
        return {"ev_m_resin": sc["Mr"], "ev_m_solvent": 1.0, "ev_e0": 1.0, "ev_power_n": ev.get("PowerN", 0.5),
                "ev_negpow_exp": ev.get("NegPowExponent", 0.25),
                "ev_negpow_rmax": ev.get("NegPowRmax", 75e-3) / sc["L0"], "ev_conc_r": ev.get("ConcR", 0.0),
                "ev_h_ast": self.precursor, "evap_hast_modify": int(self.precursor != 0.0)}

    # ------------------------------------------------------------------
    def write_fields(self, path, h, c) -> None:
        """h, c (and this case's substrate s) on the whole grid (nx*ny) as an
        ASCII field file of the reference's restart (columns x y h+s u v c h
        s, rows of grid points 1..nx-2 x 1..ny-2, iy outer, non-dimensional)."""
        _, _, s = self.fields()
        nx, ny = self.Nx + 4, self.Ny + 4
        lines = ["# x y h+s u v c h s"]
        for iy in range(1, ny - 1):
            for ix in range(1, nx - 1):
                i = iy * nx + ix
                hi, ci, si = float(h[i]), float(c[i]), float(s[i])
                lines.append(f"{float(ix)!r} {float(iy)!r} {hi + si!r} 0.0 0.0 {ci!r} {hi!r} {si!r}")
        Path(path).write_text("\n".join(lines) + "\n")

    def write_reference(self, workdir) -> Path:
        """case.toml and the ASCII restart init.dat (columns x y h+s u v c h s,
        rows of grid points 1..nx-2 x 1..ny-2, iy outer; non-dimensional,
        read with coefficient 1 as Output.Dimensioned = false makes it)."""
        w = Path(workdir)
        w.mkdir(parents=True, exist_ok=True)
        h, c, _ = self.fields()
        self.write_fields(w / "init.dat", h, c)
        (w / "case.toml").write_text(toml_dumps(self.toml("init.dat")))
        return w / "case.toml"


# ----------------------------------------------------------------------
#  the benchmark workloads (seeded synthetic inputs)
# ----------------------------------------------------------------------
def spinodal_224(N: int = 224, seed: int = 20261203, steps: int = 12, end_time: float = 0.8) -> Case:
    """Spinodal dewetting of a periodic 224^2 film, capillary + disjoining
    pressure, theta_e = 10 deg, h* = 0.01 h0, h = 1 + 1e-3 U(-1, 1), adaptive dt."""
    rng = np.random.default_rng(seed)
    h = 1.0 + 1e-3 * rng.uniform(-1.0, 1.0, size=(N, N))
    side = 0.64e-3
    return Case(name=f"spinodal_{N}", Nx=N, Ny=N, xlim=(-side / 2, side / 2), ylim=(-side / 2, side / 2),
                h0=1e-6, precursor=0.01, bc=("Periodic",) * 4, dt=1e-4, steps=steps, end_time=end_time,
                dt_control=True, disjoining=(10.0, 3.0, 2.0), h_init=h, conc0=0.5)


def dewetting(N: int, theta_e: float, amp: float, seed: int, steps: int = 12, end_time: float = 0.8) -> Case:
    """One instance of the batched ensemble: the spinodal film of
    spinodal_224 on N x N periodic cells of the same size (2.857 um), with
    contact angle theta_e [deg] and noise h = 1 + amp U(-1, 1) from its seed;
    capillary + disjoining pressure, adaptive dt."""
    rng = np.random.default_rng(seed)
    h = 1.0 + amp * rng.uniform(-1.0, 1.0, size=(N, N))
    side = 0.64e-3 * N / 224.0
    return Case(name=f"dewetting_{N}_{seed}", Nx=N, Ny=N, xlim=(-side / 2, side / 2), ylim=(-side / 2, side / 2),
                h0=1e-6, precursor=0.01, bc=("Periodic",) * 4, dt=1e-4, steps=steps, end_time=end_time,
                dt_control=True, disjoining=(theta_e, 3.0, 2.0), h_init=h, conc0=0.5)


def levelling(N: int, amp: float, waves: int, seed: int, steps: int = 12, end_time: float = 0.8) -> Case:
    """A levelling instance of the batched ensemble: a film of mean height 1
    corrugated by amp cos(pi waves (i + 1/2) / N) cos(pi waves (j + 1/2) / N)
    (a mode the mirror edges keep) with seeded noise of amp / 10, on N x N
    cells of the dewetting instances' size with Symmetry edges; capillary
    pressure and vertical gravity (the reference's leveling cases), adaptive
    dt."""
    rng = np.random.default_rng(seed)
    i = (np.arange(N) + 0.5) / N
    mode = np.outer(np.cos(math.pi * waves * i), np.cos(math.pi * waves * i))
    h = 1.0 + amp * mode + 0.1 * amp * rng.uniform(-1.0, 1.0, size=(N, N))
    side = 0.64e-3 * N / 224.0
    return Case(name=f"levelling_{N}_{seed}", Nx=N, Ny=N, xlim=(-side / 2, side / 2), ylim=(-side / 2, side / 2),
                h0=1e-6, precursor=0.01, bc=("Symmetry",) * 4, dt=1e-4, steps=steps, end_time=end_time,
                dt_control=True, vgrav=9.8, h_init=h, conc0=0.5)


def batch(count: int = 256, seed: int = 20261204, sizes=(64, 96, 128, 192, 256), steps: int = 12) -> list:
    """The batched ensemble: count seeded instances, N uniform in sizes, half
    of them (by a seeded draw) dewetting films -- theta_e uniform in [5, 20]
    deg, noise amplitude log-uniform in [1e-4, 1e-2], periodic edges -- and
    half levelling films -- corrugation amplitude log-uniform in [1e-2, 1e-1],
    one to four half-waves, mirror edges; instance k is seeded by (seed, k)."""
    rng = np.random.default_rng(seed)
    Ns = rng.choice(np.asarray(sizes), size=count)
    th = rng.uniform(5.0, 20.0, size=count)
    amp = 10.0 ** rng.uniform(-4.0, -2.0, size=count)
    kind = rng.random(size=count) < 0.5
    lamp = 10.0 ** rng.uniform(-2.0, -1.0, size=count)
    waves = rng.integers(1, 5, size=count)
    out = []
    for k in range(count):
        if kind[k]:
            out.append(levelling(int(Ns[k]), float(lamp[k]), int(waves[k]), seed=seed * 1000 + k, steps=steps))
        else:
            out.append(dewetting(int(Ns[k]), float(th[k]), float(amp[k]), seed=seed * 1000 + k, steps=steps))
    return out


def allphys(N: int = 512, steps: int = 12, dt: float = 1e-5) -> Case:
    """The all-physics film: every term of the well-mixed model on an N x N film with
    Symmetry edges.  A film edge along a 30 degree oblique tanh front
    (h = 1 behind it, the precursor 0.01 ahead, the front 8 cells wide),
    Bo = 0.5, Pg = (0.2, 0.1), Sp = 0.3 about the centre, As Ma = 0.05,
    Ev = 1e-3, Navier slip lambda = 0.05, the disjoining pressure with
    theta_e = 10 deg, and the concentration solved (WM) from c0 = 0.2 with
    mu(c) = exp(4c).  The dimensional inputs are chosen so that the reference's
    NonDimensionalNumbers::Build gives those groups (to rounding), with the
    custom length scale L0 = 100 um, h0 = 1 um; the cell is 5/512 L0 at every
    N (the domain grows with N), so that smaller N are the same film on fewer
    cells.  dt is fixed (seconds): at 1e-5 s the Newton iteration takes 4-5
    passes per step, the fewest this film takes at any dt (4.5 per step from
    1e-7 s to 1e-5 s, more above)."""
    L0, h0, sig0, rho, mu0 = 1e-4, 1e-6, 30.0e-3, 1000.0, 100.0e-3
    eps = h0 / L0
    As = (L0 / h0) ** 2
    T0 = mu0 * L0 ** 4 / (sig0 * h0 ** 3)
    g_z = 0.5 * sig0 / (rho * L0 ** 2)
    g_xy = (0.2 * sig0 * eps / (rho * L0 ** 2), 0.1 * sig0 * eps / (rho * L0 ** 2))
    omega = math.sqrt(0.3 * sig0 * h0 / (rho * L0 ** 4))
    dx = 5.0 / 512.0
    half = 0.5 * N * dx * L0
    xs = (np.arange(N) + 0.5) * dx - 0.5 * N * dx
    X, Y = np.meshgrid(xs, xs)
    s = X * math.cos(math.pi / 6.0) + Y * math.sin(math.pi / 6.0)
    prec = 0.01
    h = prec + (1.0 - prec) * 0.5 * (1.0 - np.tanh(s / (4.0 * dx)))
    fluid = {"rho": rho, "sigma": sig0, "sigma_c0": 0.2, "sigma_coef": 0.05 / As * sig0,
             "mu": mu0, "mu_c0": 0.0, "mu_exp": 4.0, "D": 1e-11, "D_c0": 0.2, "D_exp": 0.0,
             "M_solvent": 100.0, "M_resin": 2000.0}
    return Case(name=f"allphys_{N}", Nx=N, Ny=N, xlim=(-half, half), ylim=(-half, half), h0=h0, precursor=prec,
                bc=("Symmetry",) * 4, dt=dt, steps=steps, dt_control=False, fluid=fluid, length_scale=L0,
                vgrav=g_z, hgrav=g_xy, centrifugal=(omega, (0.0, 0.0)), marangoni=True,
                disjoining=(10.0, 3.0, 2.0), evaporation={"Coef": 1e-3 * h0 / T0}, slip=0.05 * h0,
                conc_model="WM", conc0=0.2, h_init=h)


def _ellipse_bump(x, y, center, width, slope):
    """C_EllipseBump of height 1 (ShapeFunctions.cpp:61-66): the profile
    RectProfile_base(rr, 0, 1, slope) (:19-22) of the elliptic radius rr,
    with Math::Sigmoid (MyMath_I.h:109-112)."""
    rr = np.sqrt(np.power((x - center[0]) / width[0], 2.0) + np.power((y - center[1]) / width[1], 2.0))

    def sig(v, v0, eps):
        return 1.0 / (1.0 + np.exp(-(v - v0) / eps))

    return sig(rr, -0.5, slope * 0.1) * (1.0 - sig(rr, 0.5, slope * 0.1))


def bench2d_512(N: int = 512, steps: int = 12) -> Case:
    """The reference's own 2-D scaling benchmark at 512^2 (cases/scaling/
    bench2d_n0512.toml, the case of its published CPU timings): a 10 um film
    of the default resist (mu(c) = exp(10 (c - 0.5)), sigma(c), D(c)) on a
    1 mm square with Symmetry edges, over a substrate step -- an elliptic bump
    of half the film's height centred at x = 0.5 mm, width 1 x 0.5 mm, edge
    0.1 mm, added to both the substrate and the free surface (stacked on a
    precursor of half the height) -- with capillary pressure, Marangoni
    stress, Raoult evaporation (1e-7 m/s) and the well-mixed concentration
    solved from c = 0.5; fixed dt = 1.25e-5 s, 12 steps.  The film and
    substrate are the reference's C_InitialSurface / C_Substrate profiles
    (InitialCondition.cpp:93-120, Substrate.cpp:48-62) restated here and
    handed to both the reference and the device through the same ASCII
    restart, so both solve the same case."""
    side = 1.0e-3
    h0 = 10e-6
    prec = 0.5
    probe = Case(name="probe", Nx=N, Ny=N, xlim=(-side / 2, side / 2), ylim=(-side / 2, side / 2), h0=h0,
                 precursor=prec, bc=("Symmetry",) * 4, dt=1.25e-5)
    L0 = probe.scales()["L0"]
    g = probe.grid(L0)
    xs = (g["xmin"] + (np.arange(N) + 2) * g["dx"] + g["dx"] * 0.5) * L0
    ys = (g["ymin"] + (np.arange(N) + 2) * g["dy"] + g["dy"] * 0.5) * L0
    X, Y = np.meshgrid(xs, ys)
    prof = _ellipse_bump(X, Y, (0.5, 0.0), (1.0, 0.5), 0.1e-3)
    #  the free surface: the bump stacked (Height 0.5, Base 0) on the
    #  precursor; the substrate: the same bump added (TotalHeight 10 um)
    hs = h0 * ((0.5 * prof) * (1.0 - prec) + prec)
    ss = h0 * np.maximum(0.0, 0.5 * prof)
    hh = np.maximum(hs - ss, prec * h0)
    return Case(name=f"bench2d_{N}", Nx=N, Ny=N, xlim=(-side / 2, side / 2), ylim=(-side / 2, side / 2), h0=h0,
                precursor=prec, bc=("Symmetry",) * 4, dt=1.25e-5, steps=steps, dt_control=False, marangoni=True,
                evaporation={"Coef": 1e-7, "ConcFunc": "Raoult", "SpatialFunc": "uniform"}, conc_model="WM",
                conc0=0.5, h_init=hh / h0, s_init=ss / h0)


CONFIGS = {"spinodal_224": spinodal_224, "allphys_512": allphys, "bench2d_512": bench2d_512}


# ----------------------------------------------------------------------
#  the ConcZ model (the film with its concentration through the thickness)
# ----------------------------------------------------------------------
@dataclass
class CzCase:
    """A 2-D ConcZ case: the film of a well-mixed Case (its fluid, physics,
    grid and non-dimensional groups, NonDimensionalNumbers::Build) with Nz
    levels through the film and the concentration equation of the CZ model.
    The seeded film replaces the one the case builds (the reference's CZ
    model reads no 2-D restart: oracle/probe/yz_probe_cz takes it as init=)."""
    base: Case
    Nz: int
    conc_linear: dict = field(default_factory=lambda: {"maxit": 5000, "eps": 1e-13, "precond": "ILU",
                                                       "scaling": True})

    def toml(self) -> dict:
        b = self.base
        doc = b.toml()
        doc["Grid"]["Nz"] = self.Nz
        doc["Physics"]["ConcField"]["Model"] = "CZ"
        doc["Restart"] = {"Enable": False}
        #  the CZ film has no upwinded term (CheckParameters refuses the key)
        del doc["Numerics"]["Convection"]["Height"]
        cl = self.conc_linear
        doc["Numerics"]["ConcEquation"]["LinearSolver"] = {
            "Backend": "amgcl", "MaxIterations": cl["maxit"], "Epsilon": cl["eps"], "RowScaling": cl["scaling"],
            "PreconditionType": cl["precond"]}
        return doc

    def zeta(self) -> float:
        """C_Grid3D::Build (Grids.cpp:150-183) with RectGrid::SetExtentZ: the
        spacing of the zeta levels with two ghost levels at each end."""
        d0 = (1.0 - 0.0) / float(self.Nz)
        zmin, zmax = 0.0 - 2 * d0, 1.0 + 2 * d0
        return (zmax - zmin) / (self.Nz + 4)

    def record(self) -> dict:
        """The model's state as the reference's Build leaves it, in the keys of
        oracle/probe/yz_probe_cz (yuzen_b200.cz.params_from_record)."""
        b = self.base
        sc = b.scales()
        g = b.grid(sc["L0"])
        ev = b.evaporation or {}
        f = b.fluid
        nx, ny, nz = g["nx"], g["ny"], self.Nz + 4
        dt = b.dt / sc["T0"]
        #  C_TimeSteps::Build's range (TimeSteps.cpp:38-60), capped by the
        #  output intervals in ConcZ_Model_2D::Run (:714-735)
        dt_max = 1e10
        cap = 1e30 / sc["T0"]
        if cap < dt_max:
            dt_max = cap
        if dt_max < dt:
            dt = dt_max
        h, c, s = b.fields()
        evp = b._evap_params(sc)
        xc = [g["xmin"] + ix * g["dx"] + g["dx"] * 0.5 for ix in range(nx)]
        xf = [g["xmin"] + ix * g["dx"] + 0.0 for ix in range(nx)]
        yc = [g["ymin"] + iy * g["dy"] + g["dy"] * 0.5 for iy in range(ny)]
        yf = [g["ymin"] + iy * g["dy"] + 0.0 for iy in range(ny)]
        lin, cl = b.linear, self.conc_linear
        pre = {"None": 0, "Jacobi": 1, "ILU": 2}
        #  without the control the solver keeps C_ImplicitSolver's defaults
        dtc = b.dtc if b.dt_control else {"KeepSteps": 50, "ChangeFactor": 0.5, "Criterion": 1e-3, "ScaleFloor": 0.0}
        rec = {
            "nx": nx, "ny": ny, "nz": nz, "bc": np.array([BC[x] for x in b.bc], np.int32),
            "on_lap": int(b.laplace), "on_sc": int(b.marangoni), "on_vg": int(b.vgrav is not None),
            "on_hg": int(b.hgrav is not None), "on_cf": int(b.centrifugal is not None),
            "on_evap": int(b.evaporation is not None), "on_mms": 0,
            "ev_conc": 1 if ev.get("ConcFunc") == "PowerN" else 0,
            "ev_spatial": 1 if ev.get("SpatialFunc") == "negPow" else 0,
            "ev_hast": evp["evap_hast_modify"], "dt_control": int(b.dt_control), "dt_keep_steps": dtc["KeepSteps"],
            "max_steps": b.steps,
            "h_lin": np.array([pre[lin["precond"]], int(lin["scaling"]), lin["maxit"], 0], np.int32),
            "c_lin": np.array([pre[cl["precond"]], int(cl["scaling"]), cl["maxit"], 1], np.int32),
            "c_scheme": SCHEMES[b.conv_conc],
            "dx": g["dx"], "dy": g["dy"], "dzeta": self.zeta(), "theta_h": 0.5, "theta_c": 0.5,
            "dt": dt, "dt_old": dt, "dt_max": dt_max, "dt_min": 1e-15, "time": 0.0,
            "dt_change_factor": dtc["ChangeFactor"], "dt_criterion": dtc["Criterion"],
            "dt_scale_floor": dtc["ScaleFloor"],
            "As": sc["As"], "Ma": sc["Ma"], "Bo": sc["Bo"], "Pgx": sc["Pgx"], "Pgy": sc["Pgy"], "Sp": sc["Sp"],
            "Df": sc["Df"], "Ev": sc["Ev"],
            "rot_center": np.array([(b.centrifugal[1][0] if b.centrifugal else 0.0) / sc["L0"],
                                    (b.centrifugal[1][1] if b.centrifugal else 0.0) / sc["L0"]]),
            "visc": np.array([f["mu_c0"], 1.0, f["mu_exp"]]), "sigma": np.array([f["sigma_c0"], 1.0, sc["Ma"]]),
            "diff": np.array([f["D_c0"], 1.0, f["D_exp"]]),
            "evap": np.array([evp["ev_m_resin"], evp["ev_m_solvent"], evp["ev_e0"], evp["ev_power_n"],
                              evp["ev_negpow_exp"], evp["ev_negpow_rmax"], evp["ev_conc_r"], evp["ev_h_ast"],
                              min(g["dx"], g["dy"])]),
            "h_eps": lin["eps"], "c_eps": cl["eps"], "coupling_floor": max(1e-10, 10.0 * cl["eps"]),
            "xc": np.array(xc), "xf": np.array(xf), "yc": np.array(yc), "yf": np.array(yf),
            "h0": h, "s": s, "c0": np.full(nx * ny * nz, float(b.conc0)),
        }
        return rec

    def write_reference(self, workdir) -> Path:
        """case.toml and init.bin (the film, nx*ny doubles, row iy*nx + ix,
        ghosts included) for oracle/probe/yz_probe_cz ... init=init.bin."""
        w = Path(workdir)
        w.mkdir(parents=True, exist_ok=True)
        h, _, _ = self.base.fields()
        np.asarray(h, "<f8").tofile(w / "init.bin")
        (w / "case.toml").write_text(toml_dumps(self.toml()))
        return w / "case.toml"


def cz_bumps(N: int = 256, Nz: int = 16, seed: int = 20261205, steps: int = 6, dt: float = 0.01,
             bumps: int = 8, sigma_cells: float = 10.0, amp: float = 0.05, Ev: float = 2e-3, Df: float = 1.0,
             conc0: float = 0.3, side: float = 1.0e-3) -> CzCase:
    """The evaporating film through the thickness at N^2 x Nz: h = 1 +
    amp * the sum of `bumps` Gaussians of sigma_cells cells at seeded
    centres, c = conc0, capillary + Marangoni + evaporation, mu(c), sigma(c)
    and D(c) of the reference's resist (concz_2d.toml), Symmetry edges, a
    fixed dt [s]; the evaporation coefficient and the diffusivity chosen so
    that Ev and Df come out as given (T0 = mu L0^4 / (sigma h0^3))."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0, N, bumps), rng.uniform(0, N, bumps)
    ii = np.arange(N) + 0.5
    X, Y = np.meshgrid(ii, ii)
    h = np.ones((N, N))
    for k in range(bumps):
        h += amp * np.exp(-((X - cx[k]) ** 2 + (Y - cy[k]) ** 2) / (2.0 * sigma_cells ** 2))
    fluid = {"rho": 1000.0, "sigma": 30.0e-3, "sigma_c0": 0.5, "sigma_coef": 10e-3,
             "mu": 100.0e-3, "mu_c0": 0.5, "mu_exp": 10.0, "D": 1.0e-9, "D_c0": 0.5, "D_exp": -7.0,
             "M_solvent": 100.0, "M_resin": 2000.0}
    h0 = 10e-6
    L0 = math.sqrt(fluid["sigma"] / (fluid["rho"] * GG))
    T0 = fluid["mu"] * math.pow(L0, 4.0) / (fluid["sigma"] * math.pow(h0, 3.0))
    fluid["D"] = Df * math.pow(L0, 2.0) / T0
    base = Case(name=f"cz_bumps_{N}", Nx=N, Ny=N, xlim=(-0.5 * side, 0.5 * side), ylim=(-0.5 * side, 0.5 * side),
                h0=h0, precursor=0.5, bc=("Symmetry",) * 4, dt=dt, steps=steps, fluid=fluid, marangoni=True,
                evaporation={"Coef": Ev * h0 / T0, "ConcFunc": "Raoult", "SpatialFunc": "uniform"},
                conc_model="CZ", conc0=conc0, h_init=h)
    return CzCase(base=base, Nz=Nz)
