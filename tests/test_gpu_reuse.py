"""The engine's reuse paths against the plain transform sequence.

With reuse on (the default) the programs take fields that are exact
consequences of earlier ones: the transport's w = u + tau d and the next
gradient's u, grad u, S, A, c and pressure source formed pointwise or from
the line search's coefficient fields, the line search's S_0 from the
gradient, and the W fields as half-gradients of the |phi|^2 spectra.
MLQ_REUSE=0 runs every program in its plain transform sequence.  The CG
trajectories (J1, tau, beta and the diagnostics) must agree to rounding."""
import pytest

import maxlq_b200 as mlq

pytestmark = pytest.mark.gpu


def _trajectory(n, prec, reuse, monkeypatch):
    monkeypatch.setenv("MLQ_REUSE", reuse)
    with mlq.MaxLq(n, 4.0, 1.0, precision=prec, optim_tol=1e-14) as c:
        c.state_load(c.seed_field(2, 2.0, n / 16))
        _, st, rec = c.state_iterate(6)
        assert st == 0
        return rec


@pytest.mark.parametrize("n,prec,tol", [(64, "fp64", 1e-10), (128, "fp64", 1e-10), (128, "mixed", 2e-5)])
def test_reuse_paths_match_plain_transform_sequence(n, prec, tol, monkeypatch):
    plain = _trajectory(n, prec, "0", monkeypatch)
    reuse = _trajectory(n, prec, "1", monkeypatch)
    assert len(plain) == len(reuse) == 6
    for a, b in zip(plain, reuse):
        for k in ("J1", "tau", "R", "norm_grad", "norm_d1", "u_norm_q"):
            assert b[k] == pytest.approx(a[k], rel=tol, abs=1e-300), (a["iter"], k)
        assert b["beta"] == pytest.approx(a["beta"], rel=tol, abs=tol), (a["iter"], "beta")
        if prec == "fp64":
            assert b["n_evals"] == a["n_evals"]
