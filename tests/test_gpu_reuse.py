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


# J1, R and the norm of u to 1e-9 (FP64), as the oracle trajectory tests; the
# step and what follows from it (beta, gradient norms) to Brent's own
# resolution of a flat minimum, 1e-7, as the oracle tests take tau
@pytest.mark.parametrize("n,prec,tol_j,tol_tau", [(64, "fp64", 1e-9, 1e-7), (128, "fp64", 1e-9, 1e-7),
                                                  (128, "mixed", 2e-5, 1e-3)])
def test_reuse_paths_match_plain_transform_sequence(n, prec, tol_j, tol_tau, monkeypatch):
    plain = _trajectory(n, prec, "0", monkeypatch)
    reuse = _trajectory(n, prec, "1", monkeypatch)
    assert len(plain) == len(reuse) == 6
    for a, b in zip(plain, reuse):
        for k in ("J1", "R", "u_norm_q"):
            assert b[k] == pytest.approx(a[k], rel=tol_j), (a["iter"], k)
        for k in ("tau", "norm_grad", "norm_d1"):
            assert b[k] == pytest.approx(a[k], rel=tol_tau), (a["iter"], k)
        assert b["beta"] == pytest.approx(a["beta"], rel=tol_tau, abs=tol_tau), (a["iter"], "beta")
