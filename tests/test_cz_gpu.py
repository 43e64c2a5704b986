"""The ConcZ model's step on the device (yz_cz_*) against the reference's own
runs of its CZ model (tests/golden/cz_*.npz, made by oracle/probe/yz_probe_cz
through tests/golden/make_golden.py):

  * the pieces of one step on the start state -- the film's matrix and
    right-hand side, its face fluxes and conservative update, the velocity
    through the film, the concentration's matrix, right-hand side and volume
    fluxes -- each within 1e-12 of the reference's largest value of it;
  * the whole run (MaxSteps steps with the reference's dt control, coupling
    passes and both linear solves): the same steps and clock, the same
    linear iteration and coupling pass counts, h and c within 1e-10
    relative L2;
  * the solute of the closed film conserved on the device as in the
    reference, and two runs bit-identical;
  * the film's solves with the learned preconditioner within 1e-8 of the
    reference's run."""
from pathlib import Path

import numpy as np
import pytest

import stateio

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
CASES = ["cz_sym_16", "cz_per_koren_16", "cz_spin_fixed_18", "cz_sym_64", "cz_min_4", "cz_vanleer_per_20"]
PARTS_CASES = ["cz_sym_16", "cz_per_koren_16", "cz_spin_fixed_18", "cz_min_4", "cz_vanleer_per_20"]


def load(name):
    return stateio.load_npz(GOLD / f"{name}.npz")


def model(d):
    from yuzen_b200 import cz
    p = cz.params_from_record(d)
    return cz.CzModel(p, d["xc"], d["xf"], d["yc"], d["yf"], d["h0"], d["s"], d["c0"])


@pytest.mark.parametrize("name", PARTS_CASES)
def test_pieces_of_a_step_match_the_reference(name):
    d = load(name)
    m = model(d)
    got = m.parts()
    m.close()
    bc = d["c_bc"].astype(bool)
    bad = []
    for k, v in got.items():
        ref = d["parts_" + k]
        if k == "c_rhs":
            # only the ghost rows' right-hand sides are the step's
            v, ref = v[bc], ref[bc]
        assert v.shape == ref.shape, k
        scale = max(np.abs(ref).max(), 1e-300)
        err = np.abs(v - ref).max() / scale
        if not err <= 1e-12:
            bad.append((k, err))
    assert not bad, bad


@pytest.mark.parametrize("name", CASES)
def test_whole_run_matches_the_reference(name):
    d = load(name)
    m = model(d)
    st = m.advance(int(d["steps_done"]))
    h, c = m.fields()
    m.close()
    assert st["steps"] == d["steps_done"]
    assert abs(st["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])
    assert abs(st["dt"] - d["dt_end"]) <= 1e-12 * abs(d["dt_end"])
    assert st["linear_iterations"] == d["linear_iterations"]
    assert st["coupling_passes"] == d["coupling_passes"]
    eh = np.linalg.norm(h - d["h1"]) / np.linalg.norm(d["h1"])
    ec = np.linalg.norm(c - d["c1"]) / np.linalg.norm(d["c1"])
    assert eh <= 1e-10 and ec <= 1e-10, (eh, ec)


def test_solute_conserved_and_runs_repeat():
    d = load("cz_sym_16")
    out = []
    for _ in range(2):
        m = model(d)
        m.advance(int(d["steps_done"]))
        out.append(m.fields())
        m.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    nx, ny, nz = d["nx"], d["ny"], d["nz"]

    def solute(h, c):
        return float((h.reshape(ny, nx)[2:-2, 2:-2] * c.reshape(nz, ny, nx)[2:-2, 2:-2, 2:-2].mean(axis=0)).sum())

    s0, s1 = solute(d["h0"], d["c0"]), solute(*out[0])
    assert abs(s1 - s0) <= 1e-11 * abs(s0)


def test_bench_size_run_matches_the_reference():
    """The ConcZ workload at its bench size, 256^2 x 16 levels
    (yuzen_b200.cases.cz_bumps), built from the seed: three steps against the
    reference's run of the same film (tests/golden/czbig_256.npz, the
    reference's sources with the correctly rounded exp the device uses): the
    same steps, clock, iteration and coupling-pass counts, the film within
    1e-10 relative L2, the column sums of c and a sample of c within 1e-10.
    Against the reference built with the libm's exp (which misrounds about
    one argument in 1,300) the film is within 1e-8: the reference's own two
    builds differ by 1.0e-9 at this size (the conditioning of the film's
    capillary system), and by 2,079 against 2,172 film iterations."""
    from yuzen_b200 import cases, cz
    ref = stateio.load_npz(GOLD / "czbig_256.npz")
    rec = cases.cz_bumps(N=256, Nz=16, steps=3).record()
    m = cz.CzModel(cz.params_from_record(rec), rec["xc"], rec["xf"], rec["yc"], rec["yf"], rec["h0"], rec["s"],
                   rec["c0"])
    st = m.advance(int(ref["steps_done"]))
    h, c = m.fields()
    m.close()
    nx, ny, nz = ref["nx"], ref["ny"], ref["nz"]
    assert st["steps"] == ref["steps_done"] and abs(st["time"] - ref["t_end"]) <= 1e-12 * ref["t_end"]
    assert st["linear_iterations"] == ref["linear_iterations"] and st["coupling_passes"] == ref["coupling_passes"]
    eh = np.linalg.norm(h - ref["h1"]) / np.linalg.norm(ref["h1"])
    cs = c.reshape(nz, ny, nx)[2:-2].sum(axis=0).ravel()
    ecs = np.linalg.norm(cs - ref["c1_colsum"]) / np.linalg.norm(ref["c1_colsum"])
    esm = np.linalg.norm(c[::61] - ref["c1_sample"]) / np.linalg.norm(ref["c1_sample"])
    assert eh <= 1e-10 and ecs <= 1e-10 and esm <= 1e-10, (eh, ecs, esm)
    el = np.linalg.norm(h - ref["h1_libm"]) / np.linalg.norm(ref["h1_libm"])
    assert el <= 1e-8, el


def test_learned_film_solves_meet_the_bar():
    """The film's solves with the learned preconditioner (yz_cz_set_learned)
    on the 64^2 x 16 film with the LTE control: the first four SA-AMG film
    solves collect up to eight (residual, V-cycle) pairs each, the film solve
    after them trains the network, and the later film solves try it first
    with SA-AMG as the fallback.  The run keeps the reference's steps, its
    clock to 1e-8 and h and c within 1e-8 of the reference's run; the stats
    show the collection, the training and the network's solves or fallbacks;
    the concentration's solves are untouched (their SPAI0 / SA-AMG path)."""
    from yuzen_b200 import learned as yl
    d = load("cz_sym_64")
    m = model(d)
    m.set_learned(yl.default_config(collect_solves=4, samples_per_solve=8, capacity=32, train_iters=150, batch=4,
                                    holdout=4, cap_factor=3.0))
    st = m.advance(int(d["steps_done"]))
    h, c = m.fields()
    m.close()
    assert st["steps"] == d["steps_done"]
    assert abs(st["time"] - d["t_end"]) <= 1e-8 * abs(d["t_end"])
    eh = np.linalg.norm(h - d["h1"]) / np.linalg.norm(d["h1"])
    ec = np.linalg.norm(c - d["c1"]) / np.linalg.norm(d["c1"])
    assert eh <= 1e-8 and ec <= 1e-8, (eh, ec)
    assert st["learned_samples"] >= 8
    assert st["learned_train_ms"] > 0 and st["learned_loss"] >= 0
    assert st["learned_solves"] + st["learned_fallbacks"] >= 1, st
    print("learned film solves:", {k: st[k] for k in st if k.startswith("learned")},
          "film iterations", st["linear_iterations"], "reference", d["linear_iterations"])
