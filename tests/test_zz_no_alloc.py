"""yz_dot_noalloc: the dot product for callers that cannot allocate device
memory (a host code that owns all device memory, or a path that must not
synchronise the device the way cudaMalloc does).  It keeps its scratch in a
static array of the library instead of an allocation; this checks it through
the C ABI against yz_dot, the entry point that allocates, bit for bit, on two
calls in a row (the shared scratch keeps the first call's contents), and that
a size beyond the array is refused before any kernel runs.

The file is named to be collected last, so that a run stopping at its first
failure has run every other test already."""
import numpy as np
import pytest

import yuzen_b200 as yz

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


@pytest.mark.parametrize("n", [0, 1, 4097, 300001, 1 << 20])
def test_noalloc_matches_allocating_dot_twice(n):
    import torch
    rng = np.random.default_rng(n + 7)
    x, y = rng.standard_normal(n), rng.standard_normal(n) * 1e3
    x2, y2 = rng.standard_normal(n), rng.standard_normal(n)
    ref1, ref2 = yz.dot(x, y), yz.dot(x2, y2)
    dx, dy, dx2, dy2 = _dev(x), _dev(y), _dev(x2), _dev(y2)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    yz.dot_noalloc(n, dx.data_ptr(), dy.data_ptr(), out.data_ptr())
    yz.dot_noalloc(n, dx2.data_ptr(), dy2.data_ptr(), out.data_ptr() + 8)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[0] == ref1 and got[1] == ref2


def test_noalloc_refuses_sizes_beyond_its_scratch():
    import torch
    big = int(yz.lib().yz_dot_noalloc_max()) + 1
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(yz.YzError, match="exceeds the maximum"):
        yz.dot_noalloc(big, out.data_ptr(), out.data_ptr(), out.data_ptr())
