"""The allocation-free dealias entry point (mlq_dealias_scalar_noalloc).

It exists for callers that cannot allocate device memory, so it takes no
context and uses a static device array for all of its scratch.  Checked
through the C ABI against the context-based mlq_dealias_scalar on two calls in
a row (the second call must not see anything left by the first), directly
against the CPU oracle's dealias_scalar, for device memory that stays the same
across calls, and for its size limit.  This file is collected last so that a
failure here stops a `-x` run only after every other test has run.
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


def test_noalloc_matches_the_oracle():
    from oracle.oracle import Oracle

    lib = mlq.load_library()
    n, order = 24, 2.0
    g = np.random.default_rng(7).standard_normal((n, n, n))
    out = g.copy()
    assert lib.mlq_dealias_scalar_noalloc(dptr(out), n, order) == 0
    ref = Oracle(n, 4.0).dealias_scalar(g, order)
    assert rel(out, ref) < 1e-12


def test_noalloc_allocates_nothing_across_calls():
    import torch

    lib = mlq.load_library()
    n = 64
    g = np.random.default_rng(3).standard_normal((n, n, n))
    torch.cuda.init()
    out = g.copy()
    assert lib.mlq_dealias_scalar_noalloc(dptr(out), n, 2.0) == 0  # module and scratch are loaded by now
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        out = g.copy()
        assert lib.mlq_dealias_scalar_noalloc(dptr(out), n, 2.0) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = mlq.load_library()
    n = 2 * 64
    g = np.zeros((n, n, n))
    assert lib.mlq_dealias_scalar_noalloc(dptr(g), n, 2.0) == MLQ_ERR_BADARG
