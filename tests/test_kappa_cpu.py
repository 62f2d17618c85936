"""The gradient check's table (kappa_test, optimization.f90:957-1129) on the
host: the library's arithmetic against a line-by-line transcription of the
reference's steps, on synthetic J values with the shapes a kappa test sees
(first-order convergence, then roundoff at small epsilon)."""
import ctypes as C

import numpy as np
import pytest

import maxlq_b200 as mlq
from maxlq_b200._capi import dptr


def _reference_table(J0, J1, inner, n=16):
    """optimization.f90:1027-1081 transcribed: kappa, best kappa, adjusted kappa."""
    k = np.zeros((n, 5))
    best, bi = np.finfo(float).max, 0
    for ii in range(1, n + 1):
        eps = 10.0 ** (-7.0 - n / 2.0 + ii)
        dJ = J1[ii - 1] - J0
        kappa = dJ / (eps * inner)
        if max(abs(kappa - 1), abs(1 / kappa - 1)) < max(abs(best - 1), abs(1 / kappa - 1)):
            best, bi = kappa, ii
        k[ii - 1] = (eps, inner, dJ, kappa, kappa)
    adj, imin, fmin = 4, 1, 9999.0
    for ii in range(1, n - (adj - 1) - 1 + 1):
        f = sum(abs(1 - k[ii + jj - 1, 4] / k[ii + jj, 4]) for jj in range(adj))
        if f < fmin:
            fmin, imin = f, ii
    f = 1.0
    for jj in range(adj):
        f *= abs(k[imin + jj - 1, 4])
    f = np.copysign(f ** (1.0 / adj), k[imin - 1, 4])
    k[:, 4] /= f
    return k, f, bi, best


# at the smallest epsilon J1 - J0 can round to 0: kappa = 0, 1/kappa = inf and
# 0/0 in the adjustment window, as in the reference's IEEE arithmetic
@pytest.mark.filterwarnings("ignore::RuntimeWarning")
@pytest.mark.parametrize("seed,inner,slope", [(0, 3.7, 0.8), (1, -2.5, -40.0), (2, 1e-3, 5.0)])
def test_kappa_table_matches_the_reference_steps(seed, inner, slope):
    lib = mlq.load_library()
    n = 16
    eps = np.empty(n)
    assert lib.mlq_kappa_epsilons(n, dptr(eps)) == 0
    assert np.allclose(eps, 10.0 ** (-7.0 - n / 2 + np.arange(1, n + 1)), rtol=1e-15, atol=0)
    rng = np.random.default_rng(seed)
    J0 = 123.456
    # J(phi + eps pert) = J0 + eps inner (1 + slope eps) + roundoff of J0
    J1 = J0 + eps * inner * (1 + slope * eps) + J0 * 1e-16 * rng.standard_normal(n)
    table = np.empty((n, 5))
    frac, best = C.c_double(0.0), C.c_double(0.0)
    bi = C.c_int(0)
    assert lib.mlq_kappa_table(J0, dptr(J1), inner, n, dptr(table), C.byref(frac), C.byref(bi), C.byref(best)) == 0
    ref, f, ib, kb = _reference_table(J0, J1, inner, n)
    assert np.allclose(table, ref, rtol=1e-14, atol=0)
    assert frac.value == pytest.approx(f, rel=1e-14)
    assert bi.value == ib and best.value == pytest.approx(kb, rel=1e-14)


def test_kappa_table_rejects_short_tables():
    lib = mlq.load_library()
    table = np.empty((4, 5))
    J1 = np.ones(4)
    assert lib.mlq_kappa_table(1.0, dptr(J1), 1.0, 4, dptr(table), None, None, None) == 8
