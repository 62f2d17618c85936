"""The line search on the device (mnbrak and Brent in a conditional CUDA
graph, optimization.f90:613-951) against the host search.  Both run the same
templates over the same trial values, so every iteration must agree bit for
bit: the bracket, the step, the number of trials, J and the new state.  The
transform branch of a trial is forced with MLQ_LS_TRANSFORM_TRIALS=1 (the
polynomial shortcut off in both searches), so that the graph's conditional
check and transform bodies run on every trial."""
import os

import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu

KEYS = ("tau_a", "tau", "tau_b", "J0", "J1", "deltaJ", "beta", "n_evals", "mnbrak_flag", "status")


def _run(n, q, precision, device, iters, transform=False, seed=0):
    env = {"MLQ_DEVICE_LS": "1" if device else "0", "MLQ_LS_TRANSFORM_TRIALS": "1" if transform else "0"}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        c = mlq.MaxLq(n, q, 1.0, precision=precision, optim_tol=1e-14)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    try:
        c.state_load(seed_field(n, seed, 2.0, 2.0))
        _, st, rec = c.state_iterate(iters)
        return rec, c.kernel_config(), c.state_store(), st
    finally:
        c.close()


@pytest.mark.parametrize("n,precision,transform", [(16, "fp64", False), (64, "fp64", False),
                                                   (64, "mixed", False), (128, "mixed", False),
                                                   (32, "fp64", True), (64, "mixed", True)])
def test_device_line_search_matches_host_search(n, precision, transform):
    iters = 5
    rd, cd, ud, sd = _run(n, 4.0, precision, True, iters, transform)
    rh, ch, uh, sh = _run(n, 4.0, precision, False, iters, transform)
    assert sd == sh == 0 and len(rd) == len(rh) == iters
    # the device search ran for every iteration, the host one for none
    assert cd["line_searches_on_device"] == iters
    assert ch["line_searches_on_device"] == 0
    if transform:
        assert cd["line_search_trials_polynomial"] == ch["line_search_trials_polynomial"] == 0
    assert cd["line_search_trials_transform"] == ch["line_search_trials_transform"]
    for a, b in zip(rd, rh):
        for k in KEYS:
            assert a[k] == b[k], (k, a[k], b[k])
    assert np.array_equal(ud, uh)


def test_device_line_search_trajectory_matches_the_oracle():
    """Eight iterations at 32^3, q = 4, FP64 with the device search: the
    trials, steps and J against the CPU restatement."""
    n, q = 32, 4.0
    o = Oracle(n, q, 1.0)
    u0 = seed_field(n, 2, 2.0, 2.0)
    uo, it_o, fl_o, rec_o = o.maxdlqdt(u0, max_iter=8, optim_tol=1e-14)
    os.environ["MLQ_DEVICE_LS"] = "1"
    try:
        c = mlq.MaxLq(n, q, 1.0, max_iter=8, optim_tol=1e-14)
    finally:
        os.environ.pop("MLQ_DEVICE_LS", None)
    uc, it_c, st_c, rec_c = c.maxdLqdt(u0)
    cfg = c.kernel_config()
    c.close()
    assert it_c == it_o == 8 and st_c == 0
    assert cfg["line_searches_on_device"] == 8
    for a, b in zip(rec_c, rec_o):
        assert a["n_evals"] == b["n_evals"]
        assert a["J1"] == pytest.approx(b["J1"], rel=1e-9)
        # Brent stops at TOL = 1e-6 relative to its bracket (optimization.f90:804)
        assert a["tau"] == pytest.approx(b["tau"], rel=1e-5)
    assert float(np.abs(uc - uo).max() / np.abs(uo).max()) < 1e-6
