"""Make the golden solve fixtures of tests/golden/*.npz.

Runs the CPU oracle -- the reference's own sources compiled by oracle/Makefile
(oracle/_ref/yuzen_oracle), with the CPU restatement of the linear-solver
backend -- on small variants of the reference's shipped cases, with the dump
hook on (YZO_DUMP_DIR), and stores a few of the linear systems it solved (the
height-equation matrix I + theta dt J, the concentration matrix, their
right-hand sides, initial guesses and the oracle's answers).

    python tests/golden/make_golden.py [--ref /root/reference]

This script needs the reference checkout (it reads cases/*.toml there) and the
built oracle; the fixtures it writes are self-contained.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile
import tomllib

import numpy as np
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))

import dumpio  # noqa: E402
import stateio  # noqa: E402
import tomlw  # noqa: E402

ORACLE = REPO / "oracle" / "_ref" / "yuzen_oracle"
PROBE = REPO / "oracle" / "_ref" / "yz_probe"

QUIET_OUTPUT = {
    "Output.FieldData.TimeInterval": 1e30,
    "Output.FieldData.NeutralFile": False,
    "Output.FieldData.VTKFile": False,
    "Output.GeneralHistory.TimeInterval": 1e30,
    "Output.CalcInfo.TimeInterval": 1e30,
    "Output.ProbeList.TimeInterval": 1e30,
}

#  name: (reference case, overrides, which dumps to keep: the first three solves
#  of a run are set-up solves of the boundary rows; the Newton systems follow)
CASES = {
    # 2-D, every term of the height equation, WM concentration; 64^2 so that
    # the AMG has more than one level (n = 68^2 > 3000)
    "allphys2d_64": ("allphys_2d_reg.toml", {
        "Grid.Nx": 64, "Grid.Ny": 64,
        "Numerics.TimeStepControl.Enable": False,
        "Numerics.InitialDt": 1e-4, "Numerics.MaxSteps": 2,
    }, [4, 5, 6, 8, 10]),
    # 2-D periodic film with the disjoining pressure (no concentration solve)
    "disjoin2d_periodic_56": ("allphys_2d_reg.toml", {
        "Grid.Nx": 56, "Grid.Ny": 56,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Boundary.YminBC.Type": "Periodic", "Boundary.YmaxBC.Type": "Periodic",
        "Physics.ConcField.Model": "None",
        "Physics.SolutoCapillarity.Enable": False, "Physics.VerticalGravity.Enable": False,
        "Physics.HorizontalGravity.Enable": False, "Physics.Centrifugal.Enable": False,
        "Physics.Evaporation.Enable": False,
        "Physics.DisjoiningPressure.Enable": True, "Physics.DisjoiningPressure.ContactAngle": 10.0,
        "Physics.DisjoiningPressure.ExponentN": 3.0, "Physics.DisjoiningPressure.ExponentM": 2.0,
        "Initial.SurfaceShape.PrecursorRatio": 0.05,
        "Numerics.TimeStepControl.Enable": False,
        "Numerics.InitialDt": 1e-4, "Numerics.MaxSteps": 1,
    }, [3, 4]),
    # 1-D capillary levelling over a substrate bump (single direct AMG level)
    "leveling1d": ("leveling_1d_reg.toml", {
        "Numerics.TimeStepControl.Enable": False,
        "Numerics.InitialDt": 1e-3, "Numerics.MaxSteps": 1,
        "Numerics.HeightEquation.LinearSolver.Backend": "amgcl",
    }, [4, 6, 8, 10]),
}


#  Whole-step cases for the probe: name: (reference case, overrides, steps,
#  index of the first Newton solve among the dumps)
_NO_UPWIND = {
    "Physics.SolutoCapillarity.Enable": False, "Physics.HorizontalGravity.Enable": False,
    "Physics.Centrifugal.Enable": False, "Physics.ConcField.Model": "None",
}
STEP_CASES = {
    # capillary + disjoining pressure, periodic edges, fixed dt
    "step_disjoin_periodic_56": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 56, "Grid.Ny": 56,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Boundary.YminBC.Type": "Periodic", "Boundary.YmaxBC.Type": "Periodic",
        "Physics.VerticalGravity.Enable": False, "Physics.Evaporation.Enable": False,
        "Physics.DisjoiningPressure.Enable": True, "Physics.DisjoiningPressure.ContactAngle": 10.0,
        "Physics.DisjoiningPressure.ExponentN": 3.0, "Physics.DisjoiningPressure.ExponentM": 2.0,
        "Initial.SurfaceShape.PrecursorRatio": 0.05,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-4,
    }, 3, 3),
    # capillary over a substrate bump + vertical gravity + evaporation +
    # Navier slip, mirror edges, c carried unchanged, fixed dt
    "step_capgrav_slip_48": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 48, "Grid.Ny": 44,
        "Physics.VerticalGravity.Enable": True, "Physics.Evaporation.Enable": True,
        "Physics.Slip.Enable": True, "Physics.Slip.Length": 5e-7,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 2e-4,
    }, 4, 3),
    # every height term with the upwinded ones (in-plane gravity, rotation,
    # Marangoni) on the Koren-limited path, c carried unchanged, fixed dt
    "step_upwind_48": ("allphys_2d_reg.toml", {
        "Physics.ConcField.Model": "None", "Grid.Nx": 48, "Grid.Ny": 44,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, 3),
    # every term and the well-mixed concentration solved in every Newton pass
    "step_wm_allphys_48": ("allphys_2d_reg.toml", {
        "Grid.Nx": 48, "Grid.Ny": 40,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-2,
    }, 3, -1),
    # the same with Navier slip, the VanLeer limiter, a Koren-limited
    # concentration and the time-step control on
    "step_wm_slip_adaptive_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.Slip.Enable": True, "Physics.Slip.Length": 5e-7,
        "Numerics.Convection.Height": "VanLeer", "Numerics.Convection.Concentration": "Koren",
        "Numerics.TimeStepControl.Enable": True, "Numerics.TimeStepControl.KeepSteps": 2,
        "Numerics.TimeStepControl.ChangeFactor": 0.75, "Numerics.InitialDt": 1e-3,
    }, 6, -1),
    # every term, the well-mixed concentration solved, and the other
    # evaporation laws: PowerN in c, the negPow spatial profile, a rate ten
    # times the case's so that the caps (half the film per step, the solvent
    # there is) take part
    "step_evap_powern_negpow_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.Evaporation.ConcFunc": "PowerN", "Physics.Evaporation.PowerN": 2.0,
        "Physics.Evaporation.SpatialFunc": "negPow", "Physics.Evaporation.Coef": 1e-6,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-2,
    }, 3, -1),
    # every height term with the upwinded ones on each unlimited scheme of
    # Numerics.Convection.Height (the fixed four-point face values,
    # FiniteDifferences.cpp:22-76, 216-226), c carried unchanged, fixed dt
    **{f"step_upwind_{s.lower()}_40": ("allphys_2d_reg.toml", {
        "Physics.ConcField.Model": "None", "Grid.Nx": 40, "Grid.Ny": 36,
        "Numerics.Convection.Height": s,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, 3) for s in ("Upwind1", "Upwind2", "Central2", "UTOPIA", "QUICK", "KK", "Central4")},
    # the well-mixed concentration solved with Navier slip and the
    # Kawamura-Kuwahara height scheme (the face fluxes the concentration and
    # the energy budget take on the unlimited path), QUICK for c
    "step_wm_kk_slip_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.Slip.Enable": True, "Physics.Slip.Length": 5e-7,
        "Numerics.Convection.Height": "KK", "Numerics.Convection.Concentration": "QUICK",
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-2,
    }, 3, -1),
    # open edges (BoundaryCondition.cpp:104-187): an Outlet at Xmin, a
    # FreshInlet at Xmax, mirror edges in y (their corners mirror in y), every
    # height term, c carried unchanged, fixed dt
    "step_outlet_inlet_40": ("allphys_2d_reg.toml", {
        "Physics.ConcField.Model": "None", "Grid.Nx": 40, "Grid.Ny": 36,
        "Boundary.XminBC.Type": "Outlet", "Boundary.XmaxBC.Type": "FreshInlet",
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, 3),
    # open edges on all four sides: every corner stencil of the reference
    # (Inlet-Outlet, Inlet-Inlet, Outlet-Outlet, Outlet-Inlet; :556-597)
    "step_open_corners_40": ("allphys_2d_reg.toml", {
        "Physics.ConcField.Model": "None", "Grid.Nx": 40, "Grid.Ny": 40,
        "Boundary.XminBC.Type": "FreshInlet", "Boundary.XmaxBC.Type": "Outlet",
        "Boundary.YminBC.Type": "Outlet", "Boundary.YmaxBC.Type": "FreshInlet",
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, 3),
    # a Pinning edge at Xmin with the film shaped down to it (an EdgeBump,
    # as the reference's property tests build one), mirror edges elsewhere,
    # every height term, c carried unchanged
    "step_pinning_40": ("allphys_2d_reg.toml", {
        "Physics.ConcField.Model": "None", "Grid.Nx": 40, "Grid.Ny": 36,
        "Boundary.XminBC.Type": "Pinning",
        "Initial.SurfaceShape.PrecursorRatio": 0.02,
        "Initial.SurfaceShape.EllipseBump.Height": 0.0,
        "Initial.SurfaceShape.EdgeBump": {"Order": 1, "CreateType": "add", "Base": 0.5, "Height": 1.0,
                                          "Location": "Xmin", "Alpha": 1.0, "InnerLength": 0.05e-3,
                                          "OuterLength": 0.15e-3},
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-4,
    }, 3, 3),
    # a Pinning edge at Ymax with periodic x edges (the Pinning-Periodic
    # corners), capillary + gravity + evaporation, adaptive dt
    "step_pinning_periodic_40": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 40, "Grid.Ny": 40,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Boundary.YmaxBC.Type": "Pinning",
        "Initial.SurfaceShape.PrecursorRatio": 0.02,
        "Initial.SurfaceShape.EllipseBump.Height": 0.0,
        "Initial.SurfaceShape.EdgeBump": {"Order": 1, "CreateType": "add", "Base": 0.5, "Height": 1.0,
                                          "Location": "Ymax", "Alpha": 1.0, "InnerLength": 0.05e-3,
                                          "OuterLength": 0.15e-3},
        "Numerics.TimeStepControl.Enable": True, "Numerics.TimeStepControl.KeepSteps": 2,
        "Numerics.TimeStepControl.ChangeFactor": 0.75, "Numerics.InitialDt": 1e-4,
    }, 4, 3),
    # the well-mixed concentration solved with open edges (its own ghost rows:
    # the FreshInlet holds the start concentration, BoundaryCondition.cpp:
    # 156-163), every term, fixed dt
    "step_wm_outlet_inlet_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 36,
        "Boundary.XminBC.Type": "Outlet", "Boundary.XmaxBC.Type": "FreshInlet",
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-2,
    }, 3, -1),
    # open edges on all four sides with the concentration (its corner stencils)
    "step_wm_open_corners_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 40,
        "Boundary.XminBC.Type": "FreshInlet", "Boundary.XmaxBC.Type": "Outlet",
        "Boundary.YminBC.Type": "Outlet", "Boundary.YmaxBC.Type": "FreshInlet",
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-2,
    }, 3, -1),
    # a Pinning edge with the concentration (copied outwards there)
    "step_wm_pinning_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 36,
        "Boundary.XminBC.Type": "Pinning",
        "Initial.SurfaceShape.PrecursorRatio": 0.02,
        "Initial.SurfaceShape.EllipseBump.Height": 0.0,
        "Initial.SurfaceShape.EdgeBump": {"Order": 1, "CreateType": "add", "Base": 0.5, "Height": 1.0,
                                          "Location": "Xmin", "Alpha": 1.0, "InnerLength": 0.05e-3,
                                          "OuterLength": 0.15e-3},
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, -1),
    # the nozzle (Physics.Source): a supply at the tip of a turning arm, its
    # angular speed ramped up, its flow rate rising with a time constant;
    # capillary + gravity + evaporation, mirror edges, fixed dt
    "step_nozzle_40": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.Source": {"Enable": True, "Radius": 0.1e-3, "InletRate": 2e-3, "Conc": 0.2,
                           "TimeConstant": 1e-4, "ArmLength": 0.25e-3, "ArmCenter": [0.0, 0.0],
                           "RotationRate": 2000.0, "StartAngle": 0.3, "RampTime": 1e-4, "PlateauTime": 1e-3,
                           "SubRegions": 6},
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-4,
    }, 4, 3),
    # the same nozzle with an Outlet edge at Xmax and the time-step control
    # on (the nozzle is evaluated at the middle of each attempt's step)
    "step_nozzle_outlet_adaptive_40": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 40, "Grid.Ny": 36,
        "Boundary.XmaxBC.Type": "Outlet",
        "Physics.Source": {"Enable": True, "Radius": 0.12e-3, "InletRate": 4e-3, "Conc": 0.2,
                           "TimeConstant": 0.0, "ArmLength": 0.2e-3, "ArmCenter": [0.1e-3, 0.0],
                           "RotationRate": 3000.0, "StartAngle": 1.0, "RampTime": 0.0, "PlateauTime": 1e-3,
                           "SubRegions": 4},
        "Numerics.TimeStepControl.Enable": True, "Numerics.TimeStepControl.KeepSteps": 2,
        "Numerics.TimeStepControl.ChangeFactor": 0.75, "Numerics.InitialDt": 1e-4,
    }, 6, 3),
    # the nozzle with the well-mixed concentration: the supplied liquid at
    # the local concentration, and at the nozzle's (ConcType "supplied")
    **{f"step_wm_nozzle_{kind}_40": ("allphys_2d_reg.toml", {
        "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.Source": {"Enable": True, "Radius": 0.1e-3, "InletRate": 2e-3, "Conc": 0.2, "ConcType": kind,
                           "TimeConstant": 1e-4, "ArmLength": 0.25e-3, "ArmCenter": [0.0, 0.0],
                           "RotationRate": 2000.0, "StartAngle": 0.3, "RampTime": 1e-4, "PlateauTime": 1e-3,
                           "SubRegions": 6},
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-3,
    }, 3, -1) for kind in ("local", "supplied")},
    # capillary + disjoining with the time-step control on
    "step_adaptive_40": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 40, "Grid.Ny": 40,
        "Physics.VerticalGravity.Enable": False, "Physics.Evaporation.Enable": False,
        "Physics.DisjoiningPressure.Enable": True, "Physics.DisjoiningPressure.ContactAngle": 15.0,
        "Physics.DisjoiningPressure.ExponentN": 3.0, "Physics.DisjoiningPressure.ExponentM": 2.0,
        "Initial.SurfaceShape.PrecursorRatio": 0.1,
        "Numerics.TimeStepControl.Enable": True, "Numerics.TimeStepControl.KeepSteps": 2,
        "Numerics.TimeStepControl.ChangeFactor": 0.75, "Numerics.InitialDt": 1e-3,
    }, 10, 3),
}


#  Whole-step cases from the seeded case builder (yuzen_b200/cases.py): name:
#  (builder name, keyword arguments)
BUILT_STEP_CASES = {
    # the all-physics film of the 512^2 workload on 64^2 cells, 3 steps
    "step_allphys_64": ("allphys", {"N": 64, "steps": 3}),
    # one instance of each kind of the batched ensemble (yuzen_b200.cases.batch)
    "step_batch_dewetting_64": ("dewetting", {"N": 64, "theta_e": 12.0, "amp": 3e-3, "seed": 11, "steps": 5}),
    "step_batch_levelling_64": ("levelling", {"N": 64, "amp": 0.05, "waves": 3, "seed": 7, "steps": 5}),
}


#  Whole-step cases at the measured workloads' sizes (yuzen_b200.cases: the
#  224^2 spinodal film, the 512^2 all-physics film): name: (builder name,
#  keyword arguments).  Their fixtures are compact (big_<name>.npz): the start
#  state is rebuilt by the builder, so the fixture keeps the probe's header
#  values, hashes of its start fields and patterns, and the fields after the
#  reference's steps.
BIG_STEP_CASES = {
    # the 224^2 spinodal film: periodic, adaptive dt, 5 steps
    "spinodal_224": ("spinodal_224", {"N": 224, "steps": 5}),
    # the 512^2 all-physics film at dt = 1e-5 s, 2 steps
    "allphys_512": ("allphys", {"N": 512, "steps": 2}),
    # the reference's own 512^2 scaling case (cases/scaling/bench2d_n0512.toml), 2 steps
    "bench2d_512": ("bench2d_512", {"N": 512, "steps": 2}),
}


#  The reference's own benchmark cases restated by the seeded builder:
#  name: (reference case file, builder name, keyword arguments).  The fixture
#  (ref_<name>.npz) keeps the start state the reference's set-up builds from
#  its own TOML (the probe, one step): header values, hashes of h and c, and
#  the substrate s, which the builder restates to rounding.
REF_CASES = {
    "bench2d_512": ("scaling/bench2d_n0512.toml", "bench2d_512", {"N": 512}),
}


#  The ConcZ model (oracle/probe/yz_probe_cz): name: (reference case,
#  overrides, whether the pieces of the first step are kept too).  Each runs
#  the reference's time loop to Numerics.MaxSteps; EndTime is far.
PROBE_CZ = REPO / "oracle" / "_ref" / "yz_probe_cz"
CZ_PARTS = ("h_A", "h_B", "h_colsrc", "h_qcapx", "h_qexpx", "h_qcapy", "h_qexpy", "h_IA", "h_qx", "h_qy", "h_end",
            "h_dtdh", "ux", "uy", "c_A", "c_B", "c_rhs", "c_react", "c_qx", "c_qy", "c_w")
CZ_CASES = {
    # the reference's 2-D case: capillary + Marangoni (the coupling passes)
    # + evaporation, Symmetry walls, the LTE control cutting a long first step
    "cz_sym_16": ("concz_2d.toml", {
        "Grid.Nx": 16, "Grid.Ny": 16, "Grid.Nz": 8, "Numerics.MaxSteps": 6,
        "Numerics.InitialDt": 1000.0, "Numerics.EndTime": 1e6,
    }, True),
    # periodic film, no Marangoni (the concentration's own two stages), both
    # gravities, the limited Koren scheme (SettleLimiter) and the negPow
    # evaporation
    "cz_per_koren_16": ("concz_2d.toml", {
        "Grid.Nx": 16, "Grid.Ny": 20, "Grid.Nz": 8, "Numerics.MaxSteps": 5,
        "Numerics.InitialDt": 1.0, "Numerics.EndTime": 1e6,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Boundary.YminBC.Type": "Periodic", "Boundary.YmaxBC.Type": "Periodic",
        "Physics.SolutoCapillarity.Enable": False, "Physics.VerticalGravity.Enable": True,
        "Physics.HorizontalGravity.Enable": True, "Numerics.Convection.Concentration": "Koren",
        "Physics.Evaporation.SpatialFunc": "negPow", "Physics.Evaporation.NegPowRmax": 0.8e-3,
    }, True),
    # the centrifugal term about an off-centre axis at a fixed step
    "cz_spin_fixed_18": ("concz_2d.toml", {
        "Grid.Nx": 18, "Grid.Ny": 16, "Grid.Nz": 9, "Numerics.MaxSteps": 4,
        "Numerics.InitialDt": 0.2, "Numerics.EndTime": 1e6, "Numerics.TimeStepControl.Enable": False,
        "Physics.Centrifugal.Enable": True, "Physics.Centrifugal.RotationAxis": [0.1e-3, -0.2e-3],
    }, True),
    # the smallest grid the model takes (4 x 4 cells, 3 levels), the VanLeer
    # limiter and the PowerN evaporation
    "cz_min_4": ("concz_2d.toml", {
        "Grid.Nx": 4, "Grid.Ny": 4, "Grid.Nz": 3, "Numerics.MaxSteps": 4,
        "Numerics.InitialDt": 1.0, "Numerics.EndTime": 1e6,
        "Numerics.Convection.Concentration": "VanLeer", "Physics.Evaporation.ConcFunc": "PowerN",
    }, True),
    # the VanLeer limiter with the Marangoni coupling passes on a periodic
    # film that is not square, the LTE control on
    "cz_vanleer_per_20": ("concz_2d.toml", {
        "Grid.Nx": 20, "Grid.Ny": 12, "Grid.Nz": 6, "Numerics.MaxSteps": 5,
        "Numerics.InitialDt": 10.0, "Numerics.EndTime": 1e6,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Numerics.Convection.Concentration": "VanLeer", "Physics.VerticalGravity.Enable": True,
    }, True),
    # 64^2 x 16 levels: more than one AMG level in both solves
    "cz_sym_64": ("concz_2d.toml", {
        "Grid.Nx": 64, "Grid.Ny": 64, "Grid.Nz": 16, "Numerics.MaxSteps": 4,
        "Numerics.InitialDt": 10.0, "Numerics.EndTime": 1e6,
    }, False),
}


#  the CZ cases written as TOML for the drop-in test of seam 3
#  (tests/test_dropin_gpu.py: the reference's driver with its CZ loop on the
#  device against the reference's own run)
CZ_DROPIN_CASES = ("cz_sym_16", "cz_per_koren_16")


#  the ConcZ workload at its bench size (yuzen_b200.cases.cz_bumps), run by
#  the reference from the builder's seeded film: compact, the end state as
#  the film, the column sums of c over the real levels and every 61st c
BIG_CZ_CASES = {"cz_256": {"N": 256, "Nz": 16, "steps": 3}}


def make_big_cz_case(name: str, work: Path, threads: int) -> dict:
    sys.path.insert(0, str(REPO))
    from yuzen_b200 import cases
    kw = BIG_CZ_CASES[name]
    case = cases.cz_bumps(**kw)
    w = work / name
    case.write_reference(w)
    env = dict(os.environ, OMP_NUM_THREADS=str(min(threads, 8)))
    res = subprocess.run([str(PROBE_CZ), "case.toml", "out.bin", "init=init.bin"], cwd=w, env=env,
                         capture_output=True, text=True, timeout=3600)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_records(w / "out.bin")
    #  the same run with the libm's exp (the reference exactly as it builds)
    res = subprocess.run([str(PROBE_CZ) + "_libm", "case.toml", "out_libm.bin", "init=init.bin"], cwd=w, env=env,
                         capture_output=True, text=True, timeout=3600)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe (libm) failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    dl = stateio.read_records(w / "out_libm.bin")
    rec = case.record()
    for k, v in rec.items():
        if not np.array_equal(np.asarray(v), np.asarray(d[k])):
            raise RuntimeError(f"{name}: the builder's {k} differs from the reference's")
    nx, ny, nz = d["nx"], d["ny"], d["nz"]
    c1 = d["c1"]
    out = {k: d[k] for k in ("nx", "ny", "nz", "steps_done", "t_end", "dt_end", "linear_iterations",
                             "coupling_passes", "h1", "wall")}
    out["c1_colsum"] = c1.reshape(nz, ny, nx)[2:-2].sum(axis=0).ravel()
    out["c1_sample"] = c1[::61].copy()
    out["h1_libm"] = dl["h1"]
    out["c1_colsum_libm"] = dl["c1"].reshape(nz, ny, nx)[2:-2].sum(axis=0).ravel()
    out["linear_iterations_libm"] = dl["linear_iterations"]
    out["h0"] = d["h0"]
    out["builder"] = name
    out["threads"] = min(threads, 8)
    return out


def make_cz_case(ref: Path, name: str, work: Path) -> dict:
    src, over, parts = CZ_CASES[name]
    case = write_case(ref, src, over, name, work)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    res = subprocess.run([str(PROBE_CZ), case.name, f"{name}.bin"], cwd=work, env=env, capture_output=True, text=True,
                         timeout=900)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_records(work / f"{name}.bin")
    if parts:
        res = subprocess.run([str(PROBE_CZ), case.name, f"{name}_parts.bin", "parts"], cwd=work, env=env,
                             capture_output=True, text=True, timeout=900)
        if res.returncode != 0:
            raise RuntimeError(f"{name}: probe (parts) failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
        p = stateio.read_records(work / f"{name}_parts.bin")
        for k in CZ_PARTS:
            d["parts_" + k] = p[k]
    d["case"] = name
    return d


def make_ref_case(ref: Path, name: str, work: Path, threads: int) -> dict:
    src, builder, kw = REF_CASES[name]
    doc = tomllib.loads((ref / "cases" / src).read_text())
    tomlw.setpath(doc, "Numerics.MaxSteps", 1)
    w = work / name
    w.mkdir()
    (w / "case.toml").write_text(tomlw.dumps(doc))
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    res = subprocess.run([str(PROBE), "case.toml", f"{name}.bin"], cwd=w, env=env, capture_output=True, text=True,
                         timeout=3600)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_state(w / f"{name}.bin")
    out = {k: d[k] for k in stateio.INT_KEYS + stateio.REAL_KEYS}
    out["builder"] = builder
    out["builder_kw"] = repr(kw)
    out["sha_field_h0"] = field_hash(d["field_h0"])
    out["sha_field_c0"] = field_hash(d["field_c0"])
    out["field_s0"] = d["field_s0"]
    out["case"] = name
    return out


def field_hash(a) -> str:
    """sha256 of an array's little-endian bytes (the fixtures' check of a
    start field or pattern they do not store)."""
    import hashlib
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()).hexdigest()


def make_big_step_case(name: str, work: Path, threads: int) -> dict:
    sys.path.insert(0, str(REPO))
    from yuzen_b200 import cases
    builder, kw = BIG_STEP_CASES[name]
    case = getattr(cases, builder)(**kw)
    w = work / name
    case.write_reference(w)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    res = subprocess.run([str(PROBE), "case.toml", f"{name}.bin"], cwd=w, env=env, capture_output=True, text=True,
                         timeout=7200)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_state(w / f"{name}.bin")
    out = {k: d[k] for k in stateio.INT_KEYS + stateio.REAL_KEYS}
    out["builder"] = builder
    out["builder_kw"] = repr(kw)
    for k in ("field_h0", "field_c0", "field_s0", "rowptr", "col", "bc", "rowptr_c", "col_c"):
        out["sha_" + k] = field_hash(d[k])
    out["field_h1"] = d["field_h1"]
    if d["conc_field"]:
        out["field_c1"] = d["field_c1"]
    out["case"] = name
    return out


#  Cases the reference's driver runs with either backend (the drop-in test):
#  written as TOML files under tests/golden/cases/
DROPIN_CASES = {
    # every term of the height equation and the WM concentration equation
    "dropin_allphys_48": ("allphys_2d_reg.toml", {
        "Grid.Nx": 48, "Grid.Ny": 40,
        "Numerics.TimeStepControl.Enable": False, "Numerics.InitialDt": 1e-4, "Numerics.MaxSteps": 3,
    }),
    "dropin_disjoin_periodic_40": ("allphys_2d_reg.toml", {
        **_NO_UPWIND, "Grid.Nx": 40, "Grid.Ny": 40,
        "Boundary.XminBC.Type": "Periodic", "Boundary.XmaxBC.Type": "Periodic",
        "Boundary.YminBC.Type": "Periodic", "Boundary.YmaxBC.Type": "Periodic",
        "Physics.VerticalGravity.Enable": False, "Physics.Evaporation.Enable": False,
        "Physics.DisjoiningPressure.Enable": True, "Physics.DisjoiningPressure.ContactAngle": 10.0,
        "Physics.DisjoiningPressure.ExponentN": 3.0, "Physics.DisjoiningPressure.ExponentM": 2.0,
        "Initial.SurfaceShape.PrecursorRatio": 0.05,
        "Numerics.TimeStepControl.Enable": True, "Numerics.InitialDt": 1e-4, "Numerics.MaxSteps": 4,
    }),
}


def write_case(ref: Path, src: str, over: dict, name: str, work: Path) -> Path:
    doc = tomllib.loads((ref / "cases" / src).read_text())
    for k, v in {**QUIET_OUTPUT, **over}.items():
        tomlw.setpath(doc, k, v)
    doc["JobName"] = name
    case = work / f"{name}.toml"
    case.write_text(tomlw.dumps(doc))
    return case


#  Whole-step cases under the reference's fault switch (YUZEN_FAULT_AMGCL,
#  LinearSolverBackend.cpp:630-645): name: (step case, the switch's k:m for
#  the reference's run, the same solve counted on the device).  The switch
#  counts the solves of the amgcl backend; the reference's set-up solves of
#  the boundary rows run on its eigen backend and are not counted, so the
#  k-th counted solve is the k-th Newton solve of the film on both sides.
FAULT_STEP_CASES = {
    # the capillary + disjoining film with the time-step control, the sixth
    # Newton solve (in the third step) broken down: the attempt fails and is
    # repeated without the extrapolated start at the same dt
    "fault_adaptive_40": ("step_adaptive_40", "6:1", (6, 1)),
    # two solves in a row broken down, the eighth and ninth: the attempt
    # without the extrapolated start fails too and the step is cut
    "fault2_adaptive_40": ("step_adaptive_40", "8:2", (8, 2)),
}


def make_step_case(ref: Path, name: str, work: Path, fault: str | None = None) -> dict:
    src, over, steps, first = STEP_CASES[name]
    case = write_case(ref, src, {**over, "Numerics.MaxSteps": steps, "Output.Energy.Enable": True}, name, work)
    dump = work / f"dump_{name}"
    dump.mkdir()
    env = dict(os.environ, YZO_DUMP_DIR=str(dump), YZO_DUMP_MAX="8", OMP_NUM_THREADS="4")
    if fault:
        env["YUZEN_FAULT_AMGCL"] = fault
    res = subprocess.run([str(PROBE), case.name, f"{name}.bin"], cwd=work, env=env, capture_output=True,
                         text=True, timeout=900)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_state(work / f"{name}.bin")
    dumps = sorted(dump.glob("solve_*.bin"))
    if first >= 0:
        sys_ = dumpio.read_dump(dumps[first])
        d["sys_values"] = sys_["values"]
        d["sys_rhs"] = sys_["rhs"]
    else:
        # the first Newton pass solves the concentration first (EveryNKLoop):
        # the first dump after the set-up solves with the concentration flag
        for f in dumps:
            sys_ = dumpio.read_dump(f)
            if sys_["conc"]:
                d["csys_values"] = sys_["values"]
                d["csys_rhs"] = sys_["rhs"]
                d["csys_x"] = sys_["x"]
                break
    d["case"] = name
    return d


def make_built_step_case(name: str, work: Path) -> dict:
    sys.path.insert(0, str(REPO))
    from yuzen_b200 import cases
    builder, kw = BUILT_STEP_CASES[name]
    case = getattr(cases, builder)(**kw)
    w = work / name
    toml_path = case.write_reference(w)
    #  the reference keeps its energy history (Output.Energy)
    doc = tomllib.loads(Path(toml_path).read_text())
    tomlw.setpath(doc, "Output.Energy.Enable", True)
    Path(toml_path).write_text(tomlw.dumps(doc))
    dump = (w / "dump").resolve()
    dump.mkdir()
    #  the restart's set-up solves of the boundary rows come first
    env = dict(os.environ, YZO_DUMP_DIR=str(dump), YZO_DUMP_MAX="64", OMP_NUM_THREADS="4")
    res = subprocess.run([str(PROBE), "case.toml", f"{name}.bin"], cwd=w, env=env, capture_output=True, text=True,
                         timeout=900)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: probe failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    d = stateio.read_state(w / f"{name}.bin")
    for f in sorted(dump.glob("solve_*.bin")):
        sys_ = dumpio.read_dump(f)
        if sys_["conc"]:
            d["csys_values"] = sys_["values"]
            d["csys_rhs"] = sys_["rhs"]
            d["csys_x"] = sys_["x"]
            break
    d["case"] = name
    return d


def make_case(ref: Path, name: str, work: Path) -> list[dict]:
    src, over, keep = CASES[name]
    doc = tomllib.loads((ref / "cases" / src).read_text())
    for k, v in {**QUIET_OUTPUT, **over}.items():
        tomlw.setpath(doc, k, v)
    doc["JobName"] = name
    case = work / f"{name}.toml"
    case.write_text(tomlw.dumps(doc))
    dump = work / f"dump_{name}"
    dump.mkdir()
    env = dict(os.environ, YZO_DUMP_DIR=str(dump), YZO_DUMP_MAX="16", OMP_NUM_THREADS="4")
    res = subprocess.run([str(ORACLE), case.name], cwd=work, env=env, capture_output=True, text=True, timeout=900)
    if res.returncode != 0:
        raise RuntimeError(f"{name}: oracle failed\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    files = sorted(dump.glob("solve_*.bin"))
    out = [dumpio.read_dump(files[j]) for j in keep if j < len(files)]
    for d in out:
        d["case"] = name
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--only", default=None)
    ap.add_argument("--big", action="store_true", help="also the compact fixtures at the workloads' sizes")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1, help="OpenMP threads of the big runs")
    a = ap.parse_args()
    if not ORACLE.exists():
        raise SystemExit(f"{ORACLE} missing: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        cases_dir = HERE / "cases"
        cases_dir.mkdir(exist_ok=True)
        for name, (src, over) in DROPIN_CASES.items():
            write_case(Path(a.ref), src, over, name, cases_dir)
            print("case", name)
        for name in CZ_DROPIN_CASES:
            src, over, _ = CZ_CASES[name]
            write_case(Path(a.ref), src, over, "czdropin_" + name, cases_dir)
            print("case", "czdropin_" + name)
        for name in STEP_CASES:
            if a.only and name != a.only:
                continue
            d = make_step_case(Path(a.ref), name, Path(tmp))
            stateio.save_npz(HERE / f"{name}.npz", d)
            print(name, d["nx"], d["ny"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name, (base, fault, dev) in FAULT_STEP_CASES.items():
            if a.only and name != a.only:
                continue
            d = make_step_case(Path(a.ref), base, Path(tmp) / name if (Path(tmp) / name).mkdir() is None else None,
                               fault=fault)
            d["case"] = name
            d["fault_reference"] = fault
            d["fault_at"], d["fault_count"] = dev
            stateio.save_npz(HERE / f"{name}.npz", d)
            print(name, d["nx"], d["ny"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name in BUILT_STEP_CASES:
            if a.only and name != a.only:
                continue
            d = make_built_step_case(name, Path(tmp))
            stateio.save_npz(HERE / f"{name}.npz", d)
            print(name, d["nx"], d["ny"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name in REF_CASES:
            if (a.only and name != a.only) or (not a.big and a.only != name):
                continue
            d = make_ref_case(Path(a.ref), name, Path(tmp), a.threads)
            stateio.save_npz(HERE / f"ref_{name}.npz", d)
            print(name, d["nx"], d["ny"])
        for name in BIG_STEP_CASES:
            if a.only and name != a.only:
                continue
            if not a.big and a.only != name:
                continue
            d = make_big_step_case(name, Path(tmp), a.threads)
            stateio.save_npz(HERE / f"big_{name}.npz", d)
            print(name, d["nx"], d["ny"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name in BIG_CZ_CASES:
            if a.only and name != a.only:
                continue
            if not a.big and a.only != name:
                continue
            d = make_big_cz_case(name, Path(tmp), a.threads)
            stateio.save_npz(HERE / f"czbig_{name.split('_')[-1]}.npz", d)
            print(name, d["nx"], d["ny"], d["nz"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name in CZ_CASES:
            if a.only and name != a.only:
                continue
            d = make_cz_case(Path(a.ref), name, Path(tmp))
            stateio.save_npz(HERE / f"{name}.npz", d)
            print(name, d["nx"], d["ny"], d["nz"], "steps", d["steps_done"], "t_end", d["t_end"])
        for name in CASES:
            if a.only and name != a.only:
                continue
            dumps = make_case(Path(a.ref), name, Path(tmp))
            dumpio.save_npz(HERE / f"solve_{name}.npz", dumps)
            print(name, [(d["n"], d["nnz"], d["conc"], d["iter"], d["ret"]) for d in dumps])


if __name__ == "__main__":
    main()
