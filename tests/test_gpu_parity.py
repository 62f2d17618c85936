"""GPU parity: the CUDA path through the C ABI against the CPU oracle and the
golden fixtures.  FP64 mode: 1e-10 relative (R, gradient); mixed mode
(FP32 fields and FFTs, FP64 reductions): 1e-5 relative."""
import glob
import os

import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "golden_*.npz")))
TOL64 = 1e-10
TOL32 = 2e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


_ctx_cache = {}


def ctx(n, q, B=1.0, precision="fp64"):
    key = (n, q, B, precision)
    if key not in _ctx_cache:
        _ctx_cache[key] = mlq.MaxLq(n, q, B, precision=precision)
    return _ctx_cache[key]


# ---- fftwfunction.f90 ----------------------------------------------------------
@pytest.mark.parametrize("n", [8, 12, 16, 24, 32, 48, 64])
def test_fft_c2c(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    c = ctx(n, 4.0)
    assert rel(c.fftfwd(a), np.fft.fftn(a)) < 1e-13
    assert rel(c.fftbwd(a), np.fft.ifftn(a)) < 1e-13


@pytest.mark.parametrize("n", [8, 12, 16, 32, 48, 64])
def test_fft_r2c_c2r(n):
    rng = np.random.default_rng(n + 1)
    u = rng.standard_normal((n, n, n))
    c = ctx(n, 4.0)
    fu = c.fftfwdr(u)
    assert rel(fu, np.fft.rfftn(u)) < 1e-13
    assert rel(c.fftbwdr(fu), u) < 1e-13


@pytest.mark.parametrize("n", [12, 16, 32])
@pytest.mark.parametrize("order", [2.0, 1.5, 3.0])
def test_dealias_scalar(n, order):
    rng = np.random.default_rng(3)
    g = rng.standard_normal((n, n, n))
    assert rel(ctx(n, 4.0).dealias_scalar(g, order), Oracle(n, 4.0).dealias_scalar(g, order)) < 1e-12


@pytest.mark.parametrize("n", [8, 12, 16])
def test_full_band_operators(n):
    """Arbitrary (not band-limited) inputs: Nyquist handling must match c2c + REAL()."""
    rng = np.random.default_rng(11)
    f = rng.standard_normal((n, n, n))
    u = rng.standard_normal((3, n, n, n))
    c, o = ctx(n, 4.0), Oracle(n, 4.0)
    assert rel(c.gradient(f), o.gradient(f)) < 1e-12
    assert rel(c.divergence(u), o.divergence(u)) < 1e-12
    assert rel(c.laplacian(u), o.laplacian(u)) < 1e-12
    assert rel(c.solve_poisson(f, 0.7), o.solve_poisson(f, 0.7)) < 1e-12


# ---- state operators against the golden fixtures -------------------------------
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p))
def test_golden(path):
    g = np.load(path)
    n, q, B = int(g["n"]), float(g["q"]), float(g["B"])
    c = ctx(n, q, B)
    u, d = g["u"], g["d"]
    assert rel(c.calc_global_dLqdt_inclParts(u), g["R_parts"]) < TOL64
    assert c.calc_global_Lq_norm(u) == pytest.approx(float(g["lq_norm"]), rel=1e-12)
    assert c.eval_J(u + 0.05 * d, "LineMin") == pytest.approx(float(g["J_linemin"]), rel=TOL64)
    grad = c.GradL2ForLq(u)
    assert rel(grad, g["grad_l2"]) < TOL64
    s = 1.5 - 1.0 / q
    assert rel(c.divAvg_free(c.HilbertGradient(grad, s)), g["divavg_hilbert"]) < TOL64
    assert rel(c.calcConstraintDerivativeL2(u), g["normal_l2"]) < TOL64
    assert rel(c.vectorTransport(u, q, B, 0.05 * d, grad), g["transport"]) < TOL64
    assert c.global_summed_field_inner_product(u, d, "H_l^(3/2-1/q)") == pytest.approx(
        float(g["inner_hl"]), rel=1e-10, abs=1e-13)
    assert c.global_summed_field_inner_product(u, d, "L2") == pytest.approx(
        float(g["inner_l2"]), rel=1e-10, abs=1e-13)
    assert rel(c.calc_uk(u, q - 2.0), g["uk_q2"]) < TOL64


# ---- seeded fields, larger N, against the oracle ------------------------------
@pytest.mark.parametrize("n,q", [(32, 4.0), (32, 3.0), (24, 6.0), (48, 4.0), (32, 8.0)])
def test_seeded_R_and_gradient(n, q):
    o = Oracle(n, q, 1.0)
    u = o.rescale(seed_field(n, 0, 2.0, n / 16))
    c = ctx(n, q)
    assert rel(c.calc_global_dLqdt_inclParts(u), o.R_parts(u)) < TOL64
    assert rel(c.GradL2ForLq(u), o.grad_l2(u)) < TOL64


@pytest.mark.parametrize("n,q", [(32, 4.0), (32, 6.0), (32, 3.0)])
def test_mixed_precision_R_and_gradient(n, q):
    o = Oracle(n, q, 1.0)
    u = o.rescale(seed_field(n, 1, 2.0, n / 16))
    c = ctx(n, q, precision="mixed")
    assert rel(c.calc_global_dLqdt_inclParts(u), o.R_parts(u)) < TOL32
    assert rel(c.GradL2ForLq(u), o.grad_l2(u)) < 50 * TOL32


def test_seed_field_matches_checker():
    n = 32
    assert rel(ctx(n, 4.0).seed_field(5, 2.0, 2.0), seed_field(n, 5, 2.0, 2.0)) < 1e-13


def test_rejects_field_outside_band():
    n = 16
    rng = np.random.default_rng(0)
    u = rng.standard_normal((3, n, n, n))
    with pytest.raises(mlq.MlqError) as e:
        ctx(n, 4.0).calc_global_dLqdt_inclParts(u)
    assert e.value.status == mlq.MLQ_ERR_NOT_BANDLIMITED


# ---- line search and the CG loop ------------------------------------------------
@pytest.mark.parametrize("q", [4.0, 3.0])
def test_mnbrak_brent(q):
    n = 16
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 2, 2.0, 2.0)))
    d = o.divavg_free(o.hilbert_gradient(o.grad_l2(u), 1.5 - 1 / q))
    d = d * np.sqrt(o.field_inner(u, u, "H") / o.field_inner(d, d, "H"))
    c = ctx(n, q)
    tb_o, fl_o = o.mnbrak(u, d, 0.0, 100.0)
    tb_c, fl_c = c.mnbrak(u, d, 0.0, 100.0)
    assert fl_o == fl_c == 0
    np.testing.assert_allclose(tb_c, tb_o, rtol=1e-9)
    t_o = o.brent(u, d, tb_o)
    t_c = c.brent(u, d, tb_c)
    assert t_c == pytest.approx(t_o, rel=1e-7)


@pytest.mark.parametrize("q", [4.0, 6.0])
def test_maxdlqdt_trajectory(q):
    n = 16
    o = Oracle(n, q, 1.0)
    u0 = seed_field(n, 0, 2.0, 2.0)
    uo, it_o, fl_o, rec_o = o.maxdlqdt(u0, max_iter=4, optim_tol=1e-14)
    c = mlq.MaxLq(n, q, 1.0, max_iter=4, optim_tol=1e-14)
    uc, it_c, st_c, rec_c = c.maxdLqdt(u0)
    c.close()
    assert it_c == it_o == 4 and st_c == 0
    for a, b in zip(rec_c, rec_o):
        assert a["n_evals"] == b["n_evals"]
        assert a["J1"] == pytest.approx(b["J1"], rel=1e-9)
        assert a["tau"] == pytest.approx(b["tau"], rel=1e-6)
        assert a["beta"] == pytest.approx(b["beta"], rel=1e-6, abs=1e-12)
    assert rel(uc, uo) < 1e-6


def test_maxdlqdt_momentum_reset_and_rolling_stop_match_the_oracle():
    """32 iterations at 16^3: beta is reset at iteration 25
    (optimization.f90:235-238) and the rolling stop (439-445: the sum of the
    last 10 relative improvements over the iteration count) ends the loop
    after iteration 32 with OPTIM_TOL = 3e-5 (its value falls from 3.9e-5 to
    2.6e-5 there, far from the threshold)."""
    n, q = 16, 4.0
    o = Oracle(n, q, 1.0)
    u0 = seed_field(n, 0, 2.0, 2.0)
    uo, it_o, fl_o, rec_o = o.maxdlqdt(u0, max_iter=40, optim_tol=3e-5)
    c = mlq.MaxLq(n, q, 1.0, max_iter=40, optim_tol=3e-5)
    uc, it_c, st_c, rec_c = c.maxdLqdt(u0)
    c.close()
    assert it_o == it_c == 32 and st_c == 0 and fl_o == 0
    assert rec_o[24]["beta"] == 0.0 and rec_c[24]["beta"] == 0.0
    assert all(r["beta"] > 0.0 for r in rec_c[1:24] + rec_c[25:])
    for a, b in zip(rec_c, rec_o):
        assert a["J1"] == pytest.approx(b["J1"], rel=1e-8)
        # Brent stops at TOL = 1e-6 relative to its bracket (optimization.f90:804)
        assert a["tau"] == pytest.approx(b["tau"], rel=1e-4)
    assert rel(uc, uo) < 1e-5


def test_taylor_gpu_matches_oracle_kappa():
    n, q = 16, 4.0
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 7, 2.0, 2.0)))
    phi = o.divavg_free(seed_field(n, 8, 2.0, 2.0))
    c = ctx(n, q)
    g = c.GradL2ForLq(u)
    ip = c.global_summed_field_inner_product(g, phi, "L2")
    J0 = c.eval_J(u)
    for h in (1e-3, 1e-5):
        kc = (c.eval_J(u + h * phi) - J0) / (h * ip)
        go = o.grad_l2(u)
        ko = (o.eval_J(u + h * phi) - o.eval_J(u)) / (h * o.field_inner(go, phi, "L2"))
        assert kc == pytest.approx(ko, rel=1e-6)
    assert abs(kc - 1.0) < 2e-3


def test_resident_state_iterations_continue_cg_memory():
    n, q = 16, 4.0
    u0 = seed_field(n, 3, 2.0, 2.0)
    a = mlq.MaxLq(n, q, 1.0, optim_tol=1e-14)
    a.state_load(u0)
    it1, st1, r1 = a.state_iterate(2)
    it2, st2, r2 = a.state_iterate(2)
    b = mlq.MaxLq(n, q, 1.0, optim_tol=1e-14)
    b.state_load(u0)
    it3, st3, r3 = b.state_iterate(4)
    assert it2 == it3 == 4
    assert [r["J1"] for r in r1 + r2] == pytest.approx([r["J1"] for r in r3], rel=1e-12)
    a.close()
    b.close()


def test_mixed_store_roundtrips_into_fp64_context():
    """Host transfers go through FP64 in both modes: a field stored by a
    mixed-precision context loads into an FP64 one."""
    n, q = 32, 4.0
    m = mlq.MaxLq(n, q, 1.0, precision="mixed")
    d = mlq.MaxLq(n, q, 1.0)
    u = m.seed_field(4, 2.0, 2.0)
    assert rel(u, seed_field(n, 4, 2.0, 2.0)) < 1e-13
    m.state_load(u)
    m.state_iterate(1)
    v = m.state_store()
    d.state_load(v)
    assert rel(d.state_store(), v) < 1e-13
    m.close()
    d.close()
