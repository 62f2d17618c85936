"""The gradient check's perturbation generators (kappa_test_pert,
function_ops.f90:615-977) on the GPU against the oracle's restatement: every
type, full-band fields, FP64.  The GPU forms each filter and divAvg_free in
one spectral pass where the reference takes a c2c round trip per step, so the
two agree to rounding (1e-11 of the field's largest value)."""
import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TYPES = [
    ("sine", (1.0, 2.0, 3.0)),
    ("divfree-sine", (2.0, 0.0, 1.0)),
    ("load-te0080", (0.0, 0.0, 0.0)),
    ("load-random-a", (0.0, 0.0, 0.0)),
    ("load-random-b", (0.0, 0.0, 0.0)),
    ("load-random-smooth-a", (0.0, 0.0, 0.0)),
    ("load-random-smooth-b", (0.0, 0.0, 0.0)),
    ("load-k-random-a", (0.5, 0.0, 0.0)),
    ("load-k-random-b", (-1.5, 0.0, 0.0)),
    ("load-random-poly-a", (-2.0, -1.0, 0.0)),
    ("load-random-poly-b", (1.5, 0.5, 0.0)),
    ("load-random-exp-a", (0.0, 0.0, 0.0)),
    ("load-random-exp-b", (0.0, 0.0, 0.0)),
    ("create-random-poly-b", (-2.0, -1.0, 0.0)),
    ("save-random", (0.0, 0.0, 0.0)),
]

_cache = {}


def _pair(n):
    if n not in _cache:
        _cache[n] = (mlq.MaxLq(n, 4.0, 1.0), Oracle(n, 4.0, 1.0))
    return _cache[n]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("n", [16, 64])
@pytest.mark.parametrize("mytype,m", TYPES)
def test_perturbation_matches_the_oracle(n, mytype, m):
    c, o = _pair(n)
    loaded = np.random.default_rng(n).standard_normal((3, n, n, n)) if mytype.startswith("load") else None
    pg, okg = c.kappa_test_pert(mytype, *m, loaded=loaded, seed=11)
    po, oko = o.kappa_test_pert(mytype, *m, loaded=loaded, seed=11)
    assert okg and oko
    if np.abs(po).max() == 0.0:
        # load-random-smooth-a below N = 21: the order-20 dealias keeps only
        # the mean, which divAvg_free removes
        assert mytype == "load-random-smooth-a" and n < 21
        assert np.abs(pg).max() < 1e-13
    else:
        assert _rel(pg, po) < 1e-11, (mytype, _rel(pg, po))


def test_load_type_without_its_file():
    """A load-* type whose file is missing: the field formed from zeros and
    successful = .false. (function_ops.f90:716-717)."""
    c, o = _pair(16)
    pg, okg = c.kappa_test_pert("load-random-poly-b", 1.0, 0.0, 0.0, loaded=None)
    po, oko = o.kappa_test_pert("load-random-poly-b", 1.0, 0.0, 0.0, loaded=None)
    assert not okg and not oko
    assert np.abs(pg).max() == 0.0 and np.abs(po).max() == 0.0


def test_unknown_type_is_an_argument_error():
    c, _ = _pair(16)
    with pytest.raises(mlq.MlqError) as e:
        c.kappa_test_pert("no-such-type")
    assert e.value.status == mlq.MLQ_ERR_BADARG


def test_random_perturbation_depends_only_on_the_seed():
    c, _ = _pair(16)
    a, _ = c.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=3)
    b, _ = c.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=3)
    d, _ = c.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, d)
