"""The CPU oracle, pinned: analytic answers, an independent transcription,
the committed golden fixtures, and the gradient's Taylor test."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from oracle.ref_numpy import RefNumpy
from oracle.seedfield import seed_field

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "golden_*.npz")))


def abc_field(n):
    """iguess = 50 (function_ops.f90:100-116)."""
    x = np.arange(n) / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    c = lambda a: np.cos(2 * np.pi * a)  # noqa: E731
    return np.stack([c(Z) + c(Y), c(X) + c(Z), c(Y) + c(X)])


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("n", [8, 12, 16])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    o = Oracle(n, 4.0)
    assert rel(o.fft_c2c(a, -1), np.fft.fftn(a)) < 1e-13
    assert rel(o.fft_c2c(a, +1), np.fft.ifftn(a)) < 1e-13


@pytest.mark.parametrize("n", [8, 16])
def test_abc_known_answer_q2(n):
    """q = 2: R = -nu ||grad u||^2 = -12 pi^2 nu for the iguess-50 field."""
    o = Oracle(n, 2.0)
    R = o.R_parts(abc_field(n))
    assert abs(R[0] - (-12.0 * np.pi ** 2)) < 1e-10
    assert R[2] == pytest.approx(0.0, abs=1e-12)


@pytest.mark.parametrize("q", [3.0, 4.0, 6.0, 8.0])
def test_oracle_matches_numpy_transcription(q):
    n = 12
    o, r = Oracle(n, q, 1.3), RefNumpy(n, q, 1.3)
    u = r.rescale(r.divavg_free(seed_field(n, 5, 2.0, 3.0)))
    d = r.divavg_free(seed_field(n, 6, 2.0, 3.0))
    assert rel(o.R_parts(u), r.R_parts(u)) < 1e-12
    assert o.lq_norm(u) == pytest.approx(r.lq_norm(u), rel=1e-13)
    g = o.grad_l2(u)
    assert rel(g, r.grad_l2(u)) < 1e-11
    assert rel(o.normal_l2(u), r.normal_l2(u)) < 1e-11
    assert rel(o.vector_transport(u, 0.1 * d, g), r.vector_transport(u, 0.1 * d, g)) < 1e-11
    assert rel(o.hilbert_gradient(g, 1.5 - 1 / q), r.hilbert(g, 1.5 - 1 / q)) < 1e-12
    assert o.field_inner(u, g, "H") == pytest.approx(r.field_inner(u, g, "H"), rel=1e-12)
    assert o.eval_J(u + 0.01 * d, "LineMin") == pytest.approx(r.eval_J(u + 0.01 * d, "LineMin"), rel=1e-12)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p))
def test_oracle_against_golden(path):
    g = np.load(path)
    n, q, B = int(g["n"]), float(g["q"]), float(g["B"])
    o = Oracle(n, q, B)
    u, d = g["u"], g["d"]
    assert rel(o.R_parts(u), g["R_parts"]) < 1e-12
    assert o.lq_norm(u) == pytest.approx(float(g["lq_norm"]), rel=1e-13)
    assert o.eval_J(u + 0.05 * d, "LineMin") == pytest.approx(float(g["J_linemin"]), rel=1e-12)
    grad = o.grad_l2(u)
    assert rel(grad, g["grad_l2"]) < 1e-11
    s = 1.5 - 1.0 / q
    assert rel(o.divavg_free(o.hilbert_gradient(grad, s)), g["divavg_hilbert"]) < 1e-11
    assert rel(o.normal_l2(u), g["normal_l2"]) < 1e-11
    assert rel(o.vector_transport(u, 0.05 * d, grad), g["transport"]) < 1e-10
    assert o.field_inner(u, d, "H") == pytest.approx(float(g["inner_hl"]), rel=1e-12, abs=1e-14)
    assert rel(o.calc_uk(u, q - 2.0), g["uk_q2"]) < 1e-12


def kappas(o, u, phi, hs=(1e-2, 1e-3, 1e-4, 1e-5)):
    g = o.grad_l2(u)
    ip = o.field_inner(g, phi, "L2")
    J0 = o.eval_J(u, "maxdLqdt")
    return [(o.eval_J(u + h * phi, "maxdLqdt") - J0) / (h * ip) for h in hs]


@pytest.mark.parametrize("q", [4.0, 6.0, 8.0])
def test_oracle_gradient_taylor(q):
    """kappa test (optimization.f90:957-1129).  The reference's L2 gradient
    is the continuous formula discretised (function_ops.f90:1192-1202), not
    the exact adjoint of the discrete R: kappa tends to 1 within ~1e-3."""
    n = 12
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 7, 2.0, 3.0)))
    phi = o.divavg_free(seed_field(n, 8, 2.0, 3.0))
    k = kappas(o, u, phi)
    assert abs(k[1] - 1) < abs(k[0] - 1)
    assert abs(k[-1] - 1.0) < 2e-3


def test_oracle_gradient_taylor_e_u_branch_is_inconsistent():
    """q < 4 takes the e_u branch; there the reference gradient is not the
    derivative of its R (kappa ~ 2): reproduced as is, not 'fixed'."""
    n = 12
    o = Oracle(n, 3.0, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 7, 2.0, 3.0)))
    phi = o.divavg_free(seed_field(n, 8, 2.0, 3.0))
    k = kappas(o, u, phi)
    assert 1.5 < k[-1] < 3.0


def test_oracle_cg_loop_increases_R():
    n, q = 12, 4.0
    o = Oracle(n, q, 1.0)
    u0 = seed_field(n, 0, 2.0, 3.0)
    u, it, flag, recs = o.maxdlqdt(u0, max_iter=3, optim_tol=1e-12)
    assert it == 3 and flag == 0
    J = [r["J1"] for r in recs]
    assert all(r["deltaJ"] >= 0 for r in recs)
    assert J[0] <= J[1] <= J[2]
    assert o.lq_norm(u) == pytest.approx(1.0, rel=1e-12)


def test_oracle_kappa_perturbations():
    """kappa_test_pert restated (function_ops.f90:615-977): the divergence-free
    sine field needs no projection, the projected types have no mean, and
    the random types depend on the seed only."""
    n = 16
    o = Oracle(n, 4.0, 1.0)
    phi, ok = o.kappa_test_pert("divfree-sine", 2.0, 0.0, 1.0)
    assert ok
    div = o.divergence(phi)
    assert np.abs(div).max() < 1e-11 * np.abs(phi).max() * 2 * np.pi * n
    a, _ = o.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=7)
    b, _ = o.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=7)
    c, _ = o.kappa_test_pert("create-random-poly-b", -2.0, -1.0, 0.0, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a.mean(axis=(1, 2, 3))).max() < 1e-14 * np.abs(a).max()
    z, ok = o.kappa_test_pert("load-k-random-a", 1.0)
    assert not ok and not z.any()
