"""Diagnostics on the GPU against the oracle: the shell spectrum
(calculate_spectral_data), the enstrophy, dEnstrophy/dt and the pointwise R
fields (calc_local_pointwise_dLqdt_inclParts), through the C ABI.
Tolerances: FP64 1e-10 relative (of the largest entry for arrays); mixed
(FP32 transforms and state) 2e-5 for the transform-based ones, 1e-6 for the
Parseval sums on the FP32 state spectra."""
import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("n,q", [(16, 4.0), (24, 3.0), (32, 6.0)])
@pytest.mark.parametrize("normalize", [True, False])
def test_spectrum(n, q, normalize):
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 1, 2.0, n / 8)))
    kk_o, sp_o = o.spectral_data(u, normalize)
    with mlq.MaxLq(n, q, 1.0) as c:
        kk_c, sp_c = c.calculate_spectral_data(u, normalize)
        c.state_load(u)
        c.state_iterate(0)  # rescale and projection only: u is already there
        kk_s, sp_s = c.calculate_spectral_data(None, normalize)
    assert np.array_equal(kk_c, kk_o)
    assert rel(sp_c, sp_o) < 1e-10
    assert rel(sp_s, sp_o) < 1e-10


@pytest.mark.parametrize("n,q", [(16, 4.0), (32, 6.0)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_enstrophy_and_its_rate(n, q, precision, tol):
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 2, 2.0, n / 8)))
    with mlq.MaxLq(n, q, 1.0, precision=precision) as c:
        ens = c.calc_global_summed_enstrophy(u)
        de = c.calc_global_dEnstrophydt(u)
    # Parseval sums on the state spectra: FP64 storage, or FP32 in the mixed path
    tol_p = 1e-10 if precision == "fp64" else 1e-6
    assert ens == pytest.approx(o.summed_enstrophy(u), rel=tol_p)
    de_o = o.dEnstrophydt(u)
    assert de[1] == pytest.approx(de_o[1], rel=tol_p)
    assert de[2] == pytest.approx(de_o[2], rel=tol, abs=tol * abs(de_o[1]))
    assert de[0] == pytest.approx(de_o[0], rel=tol, abs=tol * abs(de_o[1]))


@pytest.mark.parametrize("n,q", [(16, 4.0), (16, 3.0), (24, 6.0), (32, 8.0)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_pointwise_R(n, q, precision, tol):
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 3, 2.0, n / 8)))
    f_o = o.pointwise_R(u)
    with mlq.MaxLq(n, q, 1.0, precision=precision) as c:
        f_c = c.calc_local_pointwise_dLqdt_inclParts(u)
        R_c = c.calc_global_dLqdt_inclParts(u)
    for k in range(3):
        assert rel(f_c[k], f_o[k]) < tol, k
    # the fields integrate to R (the mean is kept by every dealias)
    assert f_c.sum(axis=(1, 2, 3)) / n**3 == pytest.approx(R_c, rel=max(tol, 1e-10), abs=1e-9 * abs(R_c[0]))
