"""The batched ensemble on the device: instances advanced concurrently
(host threads, one CUDA stream each) give every instance the film it has
when advanced alone, to the bit; a sample of the batch's instances -- one
dewetting and one levelling film, advanced among others -- ends on the
reference's own run of it (the oracle fixtures step_batch_*_64: 1e-10 on the
FP64 path, 1e-8 on the FP32 path with the autotuned launch shapes)."""
from __future__ import annotations

import numpy as np
import pytest

from yuzen_b200 import cases, ensemble
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu


def _alone(case, steps, precision=0, reuse=0):
    st0 = case.state()
    st = ys.Step(ys.params_from_state(st0), st0["field_h0"], st0["field_c0"], st0["field_s0"])
    st.set_precision(precision)
    st.set_amg_reuse(reuse)
    st.advance(steps)
    h = st.fields()[0]
    st.close()
    return h


@pytest.mark.parametrize("precision,reuse", [(0, 0), (1, 8)], ids=["fp64", "fp32_reuse"])
def test_concurrent_instances_match_each_alone(precision, reuse):
    batch = cases.batch(8, sizes=(24, 32, 40), steps=3)
    ens = ensemble.Ensemble(batch, precision=precision, amg_reuse=reuse, workers=8)
    stats = ens.advance(3)
    assert all(s["steps"] == 3 for s in stats)
    for k, c in enumerate(batch):
        assert np.array_equal(ens.fields(k)[0], _alone(c, 3, precision, reuse)), k
    ens.close()


GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"
SAMPLE = {"step_batch_dewetting_64": lambda: cases.dewetting(64, 12.0, 3e-3, seed=11, steps=5),
          "step_batch_levelling_64": lambda: cases.levelling(64, 0.05, 3, seed=7, steps=5)}


@pytest.mark.parametrize("precision,reuse,tol", [(0, 0, 1e-10), (1, 8, 1e-8)], ids=["fp64", "fp32_reuse_tuned"])
def test_sampled_instances_match_the_reference(precision, reuse, tol):
    import stateio
    from yuzen_b200 import autotune
    sample = {name: make() for name, make in SAMPLE.items()}
    others = cases.batch(6, sizes=(32, 48), steps=5)
    batch = list(sample.values()) + others
    tuning = autotune.tune(batch, precision, amg_reuse=reuse, trial=1)
    if precision:
        assert set(tuning) == {(c.Nx, c.Ny) for c in batch}
    ens = ensemble.Ensemble(batch, precision=precision, amg_reuse=reuse, workers=8, tuning=tuning)
    stats = ens.advance(5)
    for k, name in enumerate(sample):
        d = stateio.load_npz(GOLDEN / f"{name}.npz")
        h = ens.fields(k)[0]
        err = np.linalg.norm(h - d["field_h1"]) / np.linalg.norm(d["field_h1"])
        assert err <= tol, (name, err)
        assert abs(stats[k]["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"]), (name, stats[k]["time"], d["t_end"])
    ens.close()
