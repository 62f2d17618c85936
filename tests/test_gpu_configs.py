"""The workload configurations beside the headline one, at sizes a test can
afford: the 64^3 all-FP64 CG run (against the oracle on its first iteration),
a short B-continuation, and the precision/Taylor checks of the mixed path
(q = 6, B = 4, |j|^-5/3 spectrum) at 128^3.  bench.py --config c1|c2|c3 runs
them at full size."""
import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_c1_64cubed_cg_matches_oracle_then_converges():
    n, q = 64, 4.0
    u0 = seed_field(n, 0, 2.0, 4.0)
    with mlq.MaxLq(n, q, 1.0, max_iter=50, optim_tol=1e-8) as c:
        assert rel(c.seed_field(0, 2.0, 4.0), u0) < 1e-13
        u, iters, st, rec = c.maxdLqdt(u0.copy())
        assert st == mlq.MLQ_OK and 1 <= iters <= 50
        assert c.calc_global_Lq_norm(u) == pytest.approx(1.0, rel=1e-10)
        grad_scale = np.abs(c.gradient(u[0])).max()
        assert np.abs(c.divergence(u)).max() < 1e-10 * grad_scale
    R = [r["J1"] for r in rec]
    assert all(b >= a - 1e-12 * abs(a) for a, b in zip(R, R[1:]))  # R never decreases
    o = Oracle(n, q, 1.0)
    _, it_o, fl_o, rec_o = o.maxdlqdt(u0, max_iter=1, optim_tol=1e-8)
    assert rec[0]["n_evals"] == rec_o[0]["n_evals"]
    assert rec[0]["J1"] == pytest.approx(rec_o[0]["J1"], rel=1e-9)
    assert rec[0]["tau"] == pytest.approx(rec_o[0]["tau"], rel=1e-6)


def test_c2_short_b_continuation():
    n, q = 64, 4.0
    with mlq.MaxLq(n, q, 1.0, max_iter=200, optim_tol=1e-8) as c:
        u = c.seed_field(0, 2.0, 4.0)
        Rs = []
        for B in (1.0, 1.1, 1.21):
            c.set_B(B)
            u, iters, st, rec = c.maxdLqdt(u)
            assert st == mlq.MLQ_OK and iters >= 1
            assert c.calc_global_Lq_norm(u) == pytest.approx(B, rel=1e-10)
            Rs.append(c.calc_global_dLqdt_inclParts(u)[0])
    assert np.all(np.isfinite(Rs))


def test_c3_mixed_precision_errors_and_taylor_128():
    n, q, B = 128, 6.0, 4.0
    with mlq.MaxLq(n, q, B) as d, mlq.MaxLq(n, q, B, precision="mixed") as m:
        u = d.rescaleLqNorm(d.seed_field(0, 5.0 / 3.0, 16.0), B)
        phi = d.divAvg_free(d.seed_field(1, 5.0 / 3.0, 16.0))
        phi *= np.sqrt(d.global_summed_field_inner_product(u, u) / d.global_summed_field_inner_product(phi, phi))
        R_d, R_m = d.calc_global_dLqdt_inclParts(u), m.calc_global_dLqdt_inclParts(u)
        assert abs(R_m[0] - R_d[0]) / abs(R_d[0]) < 1e-6
        g_d, g_m = d.GradL2ForLq(u), m.GradL2ForLq(u)
        assert rel(g_m, g_d) < 1e-4
        ip_d = d.global_summed_field_inner_product(g_d, phi)
        ip_m = m.global_summed_field_inner_product(g_m, phi)
        err = []
        for h in (1e-2, 1e-3, 1e-4, 1e-5):
            w = u + h * phi
            kd = (d.calc_global_dLqdt_inclParts(w)[0] - R_d[0]) / (h * ip_d)
            err.append(abs(kd - 1.0))
            if h >= 1e-3:  # below, FP32 rounding of R (~1e-7 relative) dominates the difference quotient
                km = (m.calc_global_dLqdt_inclParts(w)[0] - R_m[0]) / (h * ip_m)
                assert abs(km - kd) < 2e-3 * max(1.0, abs(kd))
        # kappa(h) -> 1 linearly in h (first-order Taylor remainder)
        assert all(b < 0.2 * a for a, b in zip(err, err[1:]))
        assert err[-1] < 1e-3


def test_c4_concurrent_instances_match_one_at_a_time():
    """Independent contexts driven from several host threads at once give the
    same trajectories as the same contexts run one after another."""
    import bench

    spec = [s for s in bench.c4_instances()[:8] if s["n"] <= 64]
    ctxs = [mlq.MaxLq(s["n"], s["q"], s["B"], precision="mixed", optim_tol=0.0) for s in spec]
    fields = [c.seed_field(s["seed"], 2.0, s["n"] / 16.0) for c, s in zip(ctxs, spec)]
    _, r_seq = bench.run_instances(ctxs, fields, 2, concurrent=False)
    _, r_con = bench.run_instances(ctxs, fields, 2, concurrent=True)
    for a, b in zip(r_seq, r_con):
        assert a[1] == b[1] and len(a[2]) == len(b[2]) == 2
        assert [x["J1"] for x in a[2]] == [x["J1"] for x in b[2]]
    for c in ctxs:
        c.close()
