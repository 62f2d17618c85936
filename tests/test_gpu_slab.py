"""z-slab streaming (the memory-lean mode large N switches to) against the
resident mode on the same inputs: MLQ_SLAB_PLANES=k forces k planes per slab
for contexts created while it is set, 0 keeps every field resident."""
import numpy as np
import pytest

import maxlq_b200 as mlq

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _run(n, q, prec, planes, monkeypatch):
    monkeypatch.setenv("MLQ_SLAB_PLANES", str(planes))
    with mlq.MaxLq(n, q, 1.0, precision=prec, max_iter=3, optim_tol=1e-14) as c:
        assert c.kernel_config()["slab_planes"] == planes
        u = c.rescaleLqNorm(c.seed_field(0, 2.0, n / 16))
        out = {"R": c.calc_global_dLqdt_inclParts(u), "g": c.GradL2ForLq(u), "lq": c.calc_global_Lq_norm(u),
               "uk": c.calc_uk(u, q - 2.0)}
        out["vt"] = c.vectorTransport(u, q, 1.0, 0.01 * out["g"], out["g"])
        out["normal"] = c.calcConstraintDerivativeL2(u)
        _, it, st, rec = c.maxdLqdt(u)
        out["rec"] = rec
        f = np.random.default_rng(4).standard_normal((n, n, n))
        out["dealias"] = c.dealias_scalar(f, 2.0)
        out["grad_full"] = c.gradient(f)
    return out


@pytest.mark.parametrize("n,q,prec", [(64, 4.0, "fp64"), (64, 3.0, "fp64"), (128, 6.0, "fp64"), (64, 4.0, "mixed")])
def test_slab_mode_matches_resident_mode(n, q, prec, monkeypatch):
    a = _run(n, q, prec, 0, monkeypatch)
    b = _run(n, q, prec, 8, monkeypatch)
    tol = 1e-12 if prec == "fp64" else 2e-6
    for k in ("R", "g", "uk", "vt", "normal", "dealias", "grad_full"):
        assert rel(b[k], a[k]) < (tol if k not in ("g", "vt") or prec == "fp64" else 1e-4), k
    assert b["lq"] == pytest.approx(a["lq"], rel=tol)
    assert len(a["rec"]) == len(b["rec"]) == 3
    for x, y in zip(a["rec"], b["rec"]):
        if prec == "fp64":
            assert x["n_evals"] == y["n_evals"]
        assert y["J1"] == pytest.approx(x["J1"], rel=1e-10 if prec == "fp64" else 1e-5)
