"""The oracle's restatements of the reference's diagnostics
(calculate_spectral_data, calc_global_summed_enstrophy,
calc_global_dEnstrophydt, calc_local_pointwise_dLqdt_inclParts) against
independent numpy sums and against the oracle's own global R."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from oracle.seedfield import seed_field


def kvec(n):
    j = np.fft.fftfreq(n, 1.0 / n)
    j[n // 2] = n // 2  # the reference's Nyquist index gets +pi N
    return 2.0 * np.pi * j


@pytest.fixture(scope="module")
def case():
    n, q = 16, 4.0
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 3, 2.0, 3.0)))
    return n, q, o, u


def test_spectrum_shells_and_normalisation(case):
    n, q, o, u = case
    kk, spec = o.spectral_data(u, normalize=False)
    K = kvec(n)
    KZ, KY, KX = np.meshgrid(K, K, K, indexing="ij")
    nk = np.sqrt(KX * KX + KY * KY + KZ * KZ)
    e = sum(np.abs(np.fft.fftn(u[c])) ** 2 for c in range(3))
    ref = np.array([e[(2 * np.pi * i < nk) & (nk <= 2 * np.pi * (i + 1))].sum() for i in range(n)])
    assert np.allclose(kk, 2 * np.pi * np.arange(1, n + 1))
    assert np.abs(spec - ref).max() <= 1e-12 * ref.max()
    _, specn = o.spectral_data(u, normalize=True)
    l2 = float(np.sum(u * u)) / n**3
    assert 2 * np.pi * specn.sum() == pytest.approx(l2, rel=1e-12)


def test_enstrophy_and_its_rate_by_parseval(case):
    n, q, o, u = case
    K = kvec(n)
    KZ, KY, KX = np.meshgrid(K, K, K, indexing="ij")
    uh = [np.fft.fftn(u[c]) / n**3 for c in range(3)]
    w = [1j * (KY * uh[2] - KZ * uh[1]), 1j * (KZ * uh[0] - KX * uh[2]), 1j * (KX * uh[1] - KY * uh[0])]
    ens = 0.5 * sum(float(np.sum(np.abs(x) ** 2)) for x in w)
    assert o.summed_enstrophy(u) == pytest.approx(ens, rel=1e-12)
    k2 = KX**2 + KY**2 + KZ**2
    R1 = -float(sum(np.sum(k2**2 * np.abs(x) ** 2) for x in uh))
    out = o.dEnstrophydt(u)
    assert out[1] == pytest.approx(R1, rel=1e-12)
    assert out[0] == pytest.approx(out[1] + out[2], rel=1e-14)


@pytest.mark.parametrize("q", [4.0, 3.0, 6.0])
def test_pointwise_R_integrates_to_R(q):
    n = 12
    o = Oracle(n, q, 1.0)
    u = o.rescale(o.divavg_free(seed_field(n, 5, 2.0, 3.0)))
    f = o.pointwise_R(u)
    R = o.R_parts(u)
    dV = 1.0 / n**3
    assert f.sum(axis=(1, 2, 3)) * dV == pytest.approx(R, rel=1e-10, abs=1e-12 * abs(R[0]))
