"""Host transfers: a caller's page-locked (pinned) buffer is copied by the
DMA engine directly, a pageable one through the library's pinned staging
buffers.  Both must give the same fields bit for bit, in both precisions and
in z-slab mode."""
import numpy as np
import pytest
import torch

import maxlq_b200 as mlq

pytestmark = pytest.mark.gpu


def _pinned(a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


# 512^3 moves each field in several staging chunks (2^25 values each)
@pytest.mark.parametrize("prec,planes,n", [("fp64", 0, 64), ("mixed", 0, 64), ("mixed", 8, 64), ("mixed", 0, 512)])
def test_pinned_and_pageable_host_buffers_agree(prec, planes, n, monkeypatch):
    monkeypatch.setenv("MLQ_SLAB_PLANES", str(planes))
    with mlq.MaxLq(n, 4.0, 1.0, precision=prec, optim_tol=1e-14) as c:
        u0 = c.rescaleLqNorm(c.seed_field(3, 2.0, 4.0))
        pageable = np.ascontiguousarray(u0.copy())
        pinned, keep = _pinned(u0)
        outs = []
        for buf in (pageable, pinned):
            c.state_load(buf)
            st, _ = c.state_step(buf)
            assert st == 0
            st, _ = c.state_step(buf)
            assert st == 0
            outs.append(buf.copy())
        assert np.array_equal(outs[0], outs[1])
        g_pageable = c.GradL2ForLq(pageable)
        g_pinned = c.GradL2ForLq(pinned)
        assert np.array_equal(g_pageable, g_pinned)
        del keep
