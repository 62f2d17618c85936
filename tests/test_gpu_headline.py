"""The benchmark's workload (512^3, q = 4, seed 0, |j|^-2 exp(-(|j|/16)^2))
against the C++ oracle, through the default compile-time pass kernels.

Fixtures: tests/golden/headline_n{256,512}_q4.npz, written by
tests/golden/gen_headline.py from oracle/mlq_oracle.cpp (reference order).
Tolerances, relative:
  FP64 path   R parts 1e-10; gradient sample and norm 1e-10 (of max |grad|)
  mixed path  R 1e-6 (the stated accuracy target of the mixed path);
              gradient sample 1e-4 of max |grad|, its L2 norm 1e-5
  one CG iteration at 256^3 (the reuse paths and transform-free trials
  included): FP64 J 1e-9, tau 1e-6, same trial count; mixed J 1e-6,
  tau 1e-3.
"""
import os

import numpy as np
import pytest

import maxlq_b200 as mlq

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(n):
    p = os.path.join(HERE, f"headline_n{n}_q4.npz")
    if not os.path.exists(p):
        pytest.fail(f"missing fixture {p}: run tests/golden/gen_headline.py")
    return np.load(p)


def start_field(c, fx):
    raw = c.seed_field(int(fx["seed"]), float(fx["slope"]), float(fx["k0"]))
    return raw, c.rescaleLqNorm(c.divAvg_free(raw), float(fx["B"]))


@pytest.mark.parametrize("n", [256, 512])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_R_and_gradient_against_the_oracle(n, precision):
    fx = fixture(n)
    tol_R, tol_g, tol_gn = (1e-10, 1e-10, 1e-10) if precision == "fp64" else (1e-6, 1e-4, 1e-5)
    with mlq.MaxLq(n, float(fx["q"]), float(fx["B"]), precision=precision) as c:
        assert c.kernel_config()["pass_kernels"] == "compile-time"
        _, u = start_field(c, fx)
        R = c.calc_global_dLqdt_inclParts(u)
        v = c.GradL2ForLq(u)
    Ro = fx["R_parts"]
    assert abs(R[0] - Ro[0]) <= tol_R * abs(Ro[0])
    assert abs(R[1] - Ro[1]) <= tol_R * abs(Ro[0]) and abs(R[2] - Ro[2]) <= tol_R * abs(Ro[0])
    gs = v.ravel()[fx["grad_idx"]]
    assert np.abs(gs - fx["grad_sample"]).max() <= tol_g * float(fx["grad_maxabs"])
    gn = float(np.sqrt(np.sum(v * v) / float(n) ** 3))
    assert abs(gn - float(fx["grad_l2norm"])) <= tol_gn * float(fx["grad_l2norm"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_first_cg_iteration_at_256_against_the_oracle(precision):
    fx = fixture(256)
    tol_J, tol_tau = (1e-9, 1e-6) if precision == "fp64" else (1e-6, 1e-3)
    with mlq.MaxLq(256, float(fx["q"]), float(fx["B"]), precision=precision, max_iter=1, optim_tol=1e-14) as c:
        raw, _ = start_field(c, fx)
        _, it, st, rec = c.maxdLqdt(raw)
    assert it == 1 and st == 0
    r = rec[0]
    if precision == "fp64":
        assert r["n_evals"] == int(fx["iter1_n_evals"])
    else:
        assert abs(r["n_evals"] - int(fx["iter1_n_evals"])) <= 2
    assert r["J0"] == pytest.approx(float(fx["iter1_J0"]), rel=tol_J)
    assert r["J1"] == pytest.approx(float(fx["iter1_J1"]), rel=tol_J)
    assert r["R"] == pytest.approx(float(fx["iter1_R"]), rel=tol_J)
    assert r["tau"] == pytest.approx(float(fx["iter1_tau"]), rel=tol_tau)
