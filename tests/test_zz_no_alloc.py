"""The allocation-free dealias entry point (mlq_dealias_scalar_noalloc).

It exists for callers that cannot allocate device memory, so it takes no
context and uses a static device array for all of its scratch.  Checked
through the C ABI against the context-based mlq_dealias_scalar on two calls in
a row (the second call must not see anything left by the first), and for its
size limit.  This file is collected last so that a failure here stops a
`-x` run only after every other test has run.
"""
import numpy as np
import pytest

import maxlq_b200 as mlq
from maxlq_b200._capi import MLQ_ERR_BADARG, dptr

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("n,order", [(32, 2.0), (64, 2.0), (48, 1.5)])
def test_noalloc_matches_dealias_scalar_on_two_calls(n, order):
    lib = mlq.load_library()
    rng = np.random.default_rng(n)
    fields = [rng.standard_normal((n, n, n)), 3.0 * rng.standard_normal((n, n, n))]
    outs = []
    for g in fields:  # two calls in a row, nothing allocated in between
        out = g.copy()
        assert lib.mlq_dealias_scalar_noalloc(dptr(out), n, order) == 0
        outs.append(out)
    with mlq.MaxLq(n, 4.0) as ctx:
        refs = [ctx.dealias_scalar(g, order) for g in fields]
    for out, ref in zip(outs, refs):
        assert rel(out, ref) < 1e-12


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = mlq.load_library()
    n = 2 * 64
    g = np.zeros((n, n, n))
    assert lib.mlq_dealias_scalar_noalloc(dptr(g), n, 2.0) == MLQ_ERR_BADARG
