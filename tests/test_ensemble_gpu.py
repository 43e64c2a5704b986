"""The batched ensemble on the device: instances advanced concurrently
(host threads, one CUDA stream each) give every instance the film it has
when advanced alone, to the bit."""
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
