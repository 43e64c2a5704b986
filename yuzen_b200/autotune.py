"""The ensemble's autotuner: the shape of the FP32 V-cycle (yz_step_set_tuning)
chosen per instance size by measurement.

The coarse levels of an instance's hierarchy are a few hundred to tens of
thousands of rows, and which launch shape runs them fastest depends on the
size: whether a level's way down and way up are fused into one launch each
(and from which level), and how many lanes share a row; and how many
smoothing sweeps the finest level takes trades the cycle's cost against the
BiCGStab iterations it saves.  For each size class
of a batch the tuner takes one instance as the sample and, for every
candidate shape, builds a step context from the sample's start, runs one
untimed step (the AMG set-up, the loop graph's capture), then times `trial`
steps with CUDA events on the context's stream (yz_step_stats.device_ms); the
fastest candidate is the class's choice.  Every shape is a convergent
preconditioner of the same FP64 BiCGStab, so the instances' films meet the
FP32 forms' tolerance whichever is chosen; the FP64 cycle (the reference's)
is not tuned.

    tuning = autotune.tune(cases, precision=PREC_FP32_CYCLE, amg_reuse=64)
    ens = Ensemble(cases, precision=..., tuning=tuning)
"""
from __future__ import annotations

from . import PREC_FP64
from . import step as ys

#  (first fused level, lanes a row, finest-level sweeps): the library's
#  default (-1, 0, 0), no fusion, fusion from level 1, fixed lane counts, and
#  fewer and more sweeps
CANDIDATES = ((-1, 0, 0), (0, 0, 0), (1, 0, 0), (-1, 4, 0), (-1, 8, 0), (0, 8, 0), (-1, 0, 3), (-1, 0, 8))


def size_classes(cases) -> dict:
    """{(Nx, Ny): index of the class's first instance}."""
    out = {}
    for k, c in enumerate(cases):
        out.setdefault((c.Nx, c.Ny), k)
    return out


def time_shape(case, precision: int, amg_reuse: int, fuse_from: int, coarse_lanes: int, fine_sweeps: int = 0,
               trial: int = 2, device: int = 0, graph_loop: bool = True) -> float:
    """Device ms a step of one instance with one launch shape (after one
    untimed step)."""
    st0 = case.state()
    st = ys.Step(ys.params_from_state(st0), st0["field_h0"], st0["field_c0"], st0["field_s0"], device=device)
    try:
        st.set_precision(precision)
        st.set_amg_reuse(amg_reuse)
        st.set_graph_loop(graph_loop)
        st.set_tuning(fuse_from, coarse_lanes, fine_sweeps)
        st.advance(1)
        r = st.advance(trial)
        return float(r["device_ms"]) / max(1, trial)
    finally:
        st.close()


def tune(cases, precision: int, amg_reuse: int = 0, device: int = 0, trial: int = 2, candidates=CANDIDATES,
         graph_loop: bool = True) -> dict:
    """{(Nx, Ny): {"fuse_from", "coarse_lanes", "fine_sweeps", "ms_per_step", "default_ms_per_step",
    "trials"}} for
    every size class of cases; empty for the FP64 cycle (nothing to tune)."""
    if precision == PREC_FP64:
        return {}
    out = {}
    for size, k in sorted(size_classes(cases).items()):
        trials = {}
        for c in candidates:
            trials[c] = time_shape(cases[k], precision, amg_reuse, *c, trial=trial, device=device,
                                   graph_loop=graph_loop)
        best = min(trials, key=lambda c: (trials[c], candidates.index(c)))
        out[size] = {"fuse_from": best[0], "coarse_lanes": best[1], "fine_sweeps": best[2],
                     "ms_per_step": trials[best], "default_ms_per_step": trials.get((-1, 0, 0)),
                     "trials": {",".join(str(x) for x in c): v for c, v in trials.items()}}
    return out


def summary(tuning: dict) -> dict:
    """The choices in a JSON-friendly form: {"NxxNy": {...}}."""
    return {f"{s[0]}x{s[1]}": {k: v for k, v in t.items() if k != "trials"} for s, t in tuning.items()}
