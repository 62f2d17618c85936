"""Pass kernels specialised at compile time for power-of-two N (64 ... 1024):
against the oracle at N = 64 and 128, and at N = 256 and 512 against the
register kernels with run-time plans (MLQ_PASS_KERNELS=reg selects those for
contexts created while it is set)."""
import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("n,q", [(64, 4.0), (64, 3.0), (128, 6.0)])
def test_R_and_gradient_against_oracle(n, q):
    o = Oracle(n, q, 1.0)
    u = o.rescale(seed_field(n, 0, 2.0, n / 16))
    with mlq.MaxLq(n, q, 1.0) as c:
        R = c.calc_global_dLqdt_inclParts(u)
        g = c.GradL2ForLq(u)
    assert rel(R, o.R_parts(u)) < 1e-10
    assert rel(g, o.grad_l2(u)) < 1e-10
    with mlq.MaxLq(n, q, 1.0, precision="mixed") as m:
        assert rel(m.calc_global_dLqdt_inclParts(u), o.R_parts(u)) < 2e-5
        assert rel(m.GradL2ForLq(u), o.grad_l2(u)) < 1e-3


@pytest.mark.parametrize("n", [64, 128])
@pytest.mark.parametrize("order", [2.0, 1.5])
def test_dealias_against_oracle(n, order):
    rng = np.random.default_rng(5)
    g = rng.standard_normal((n, n, n))
    with mlq.MaxLq(n, 4.0, 1.0) as c:
        assert rel(c.dealias_scalar(g, order), Oracle(n, 4.0).dealias_scalar(g, order)) < 1e-12


def test_full_band_operators_n64():
    """Full band: the x inverse reads the Nyquist column (nx = N/2 + 1)."""
    n = 64
    rng = np.random.default_rng(12)
    f = rng.standard_normal((n, n, n))
    u = rng.standard_normal((3, n, n, n))
    o = Oracle(n, 4.0)
    with mlq.MaxLq(n, 4.0, 1.0) as c:
        assert rel(c.gradient(f), o.gradient(f)) < 1e-12
        assert rel(c.divergence(u), o.divergence(u)) < 1e-12
        assert rel(c.laplacian(u), o.laplacian(u)) < 1e-12
        assert rel(c.solve_poisson(f, 0.7), o.solve_poisson(f, 0.7)) < 1e-12


def _state_run(n, precision, kernels, monkeypatch):
    monkeypatch.setenv("MLQ_PASS_KERNELS", kernels)
    with mlq.MaxLq(n, 4.0, 1.0, precision=precision, optim_tol=1e-14) as c:
        u = c.seed_field(0, 2.0, n / 16)
        c.state_load(u)
        R, lq = c.state_R()
        g = c.GradL2ForLq(u) if n <= 256 else None
        it, st, rec = c.state_iterate(1)
    return R, lq, g, rec[0]


@pytest.mark.parametrize("n,precision,tol", [(256, "fp64", 1e-12), (256, "mixed", 2e-6), (512, "mixed", 2e-6)])
def test_compile_time_kernels_match_runtime_plan_kernels(n, precision, tol, monkeypatch):
    R0, lq0, g0, r0 = _state_run(n, precision, "reg", monkeypatch)
    R1, lq1, g1, r1 = _state_run(n, precision, "compile-time", monkeypatch)
    assert rel(R1, R0) < tol
    assert lq1 == pytest.approx(lq0, rel=tol)
    if g0 is not None:
        assert rel(g1, g0) < (tol if precision == "fp64" else 1e-4)
    if precision == "fp64":
        assert r1["n_evals"] == r0["n_evals"]  # FP32 roundoff may move Brent by an evaluation
    assert r1["J1"] == pytest.approx(r0["J1"], rel=tol)
    assert r1["tau"] == pytest.approx(r0["tau"], rel=1e-3 if precision == "mixed" else 1e-9)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gradient_graph_replay_matches_direct_launches(prec, monkeypatch):
    """The gradient program replayed as a CUDA graph gives the same CG
    trajectory, bit for bit, as the same launches issued one by one."""
    runs = {}
    for graphs in ("0", "1"):
        monkeypatch.setenv("MLQ_GRAPHS", graphs)
        with mlq.MaxLq(64, 4.0, 1.0, precision=prec, optim_tol=1e-14) as c:
            c.state_load(c.seed_field(2, 2.0, 4.0))
            _, st, rec = c.state_iterate(8)
            runs[graphs] = ([r["J1"] for r in rec], [r["tau"] for r in rec], c.kernel_config()["graph_replays"])
    assert runs["0"][0] == runs["1"][0] and runs["0"][1] == runs["1"][1]
    assert runs["0"][2] == 0 and runs["1"][2] >= 3


def _variant_run(n, precision, variant, monkeypatch):
    monkeypatch.setenv("MLQ_YZ_VARIANT", str(variant))
    with mlq.MaxLq(n, 4.0, 1.0, precision=precision, optim_tol=1e-14) as c:
        assert c.kernel_config()["yz_variants"] == f"fixed by MLQ_YZ_VARIANT={variant}"
        u = c.seed_field(1, 2.0, n / 16)
        g = c.GradL2ForLq(u)
        out = {"g": g, "uk": c.calc_uk(u, 2.0), "vt": c.vectorTransport(u, 4.0, 1.0, 0.01 * g, g)}
        f = np.random.default_rng(3).standard_normal((n, n, n))
        out["dealias"] = c.dealias_scalar(f, 2.0)
        c.state_load(u)
        out["R"] = c.state_R()[0]
        _, _, rec = c.state_iterate(2)
        out["J1"] = [r["J1"] for r in rec]
    return out


_VARIANT0 = {}


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("n,precision,tol", [(256, "fp64", 1e-12), (256, "mixed", 2e-6)])
def test_yz_tile_variants_match_default(n, precision, tol, variant, monkeypatch):
    """Every y/z tile-shape variant the autotuner may pick (including the
    column-per-warp kernels, variants 5 and 6) computes what variant 0 does:
    y and z passes both ways, z round trips, symbols and reductions."""
    if (n, precision) not in _VARIANT0:
        _VARIANT0[(n, precision)] = _variant_run(n, precision, 0, monkeypatch)
    a = _VARIANT0[(n, precision)]
    b = _variant_run(n, precision, variant, monkeypatch)
    for k in ("uk", "dealias", "R"):
        assert rel(b[k], a[k]) < tol, k
    # the gradient and the transported vector end in cancelling differences:
    # a different radix order moves them by more than the fields' roundoff
    for k in ("g", "vt"):
        assert rel(b[k], a[k]) < (1e-10 if precision == "fp64" else 1e-3), k
    assert b["J1"] == pytest.approx(a["J1"], rel=1e-10 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("variant", [5, 6])
def test_column_per_warp_variants_512_mixed(variant, monkeypatch):
    a = _state_run(512, "mixed", "compile-time", monkeypatch)
    monkeypatch.setenv("MLQ_YZ_VARIANT", str(variant))
    b = _state_run(512, "mixed", "compile-time", monkeypatch)
    assert rel(b[0], a[0]) < 2e-6
    assert b[1] == pytest.approx(a[1], rel=2e-6)
    assert b[3]["J1"] == pytest.approx(a[3]["J1"], rel=2e-6)


@pytest.mark.parametrize("variant", [8, 9])
@pytest.mark.parametrize("n", [256, 512])
def test_column_pair_y_pass_matches_default(n, variant, monkeypatch):
    """Variants 8 and 9 (two or three resident blocks), the y passes, the z
    forward (with its round trips, symbols and reductions) and the z inverse
    on column pairs (FP32 only), compute what
    variant 0 does, with an even nx (256: 86) and an odd one (512: 171, the
    pad column of the even row pitch rides in the last pair)."""
    if (n, "mixed") not in _VARIANT0:
        _VARIANT0[(n, "mixed")] = _variant_run(n, "mixed", 0, monkeypatch)
    a = _VARIANT0[(n, "mixed")]
    b = _variant_run(n, "mixed", variant, monkeypatch)
    for k in ("uk", "dealias", "R"):
        assert rel(b[k], a[k]) < 2e-6, k
    for k in ("g", "vt"):
        assert rel(b[k], a[k]) < 1e-3, k
    assert b["J1"] == pytest.approx(a["J1"], rel=1e-5)


@pytest.mark.parametrize("n,precision,variant", [(256, "fp64", None), (512, "mixed", None), (512, "mixed", "8")])
def test_multi_output_z_inverse_matches_one_output_per_launch_row(n, precision, variant, monkeypatch):
    """z inverse launches that share one source spectrum among a field and
    its derivatives (MLQ_ZMULTI, the default) give what one op per output
    gives, bit for bit: the same symbol arithmetic on the same loaded values."""
    runs = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("MLQ_ZMULTI", flag)
        if variant is None:
            monkeypatch.setenv("MLQ_AUTOTUNE", "0")
        else:  # the column-pair kernels (one-output ops of the pair kernel without grouping)
            monkeypatch.setenv("MLQ_YZ_VARIANT", variant)
        with mlq.MaxLq(n, 4.0, 1.0, precision=precision, optim_tol=1e-14) as c:
            u = c.seed_field(1, 2.0, n / 16)
            R = c.calc_global_dLqdt_inclParts(u)
            g = c.GradL2ForLq(u) if n <= 256 else None
            c.state_load(u)
            _, _, rec = c.state_iterate(2)
            runs[flag] = (R, g, [r["J1"] for r in rec], [r["tau"] for r in rec])
    a, b = runs["0"], runs["1"]
    assert np.array_equal(a[0], b[0])
    if a[1] is not None:
        assert np.array_equal(a[1], b[1])
    assert a[2] == b[2] and a[3] == b[3]


def test_fp32_state_of_the_mixed_path_tracks_its_fp64_state(monkeypatch):
    """The mixed path stores its CG state vectors in FP32 (every operation on
    them, the reductions, beta and the retraction compute in FP64); with
    MLQ_STATE_F64=1 it keeps them in FP64.  Five iterations at 256^3 agree to
    the FP32 rounding of the state: J to 1e-6, the same trial counts within
    one evaluation."""
    runs = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("MLQ_STATE_F64", flag)
        with mlq.MaxLq(256, 4.0, 1.0, precision="mixed", optim_tol=1e-14) as c:
            c.state_load(c.seed_field(0, 2.0, 8.0))
            _, st, rec = c.state_iterate(5)
            R, lq = c.state_R()
            runs[flag] = (rec, R, lq, st)
    a, b = runs["1"], runs["0"]
    assert a[3] == b[3] == 0
    for ra, rb in zip(a[0], b[0]):
        assert rb["J1"] == pytest.approx(ra["J1"], rel=1e-6)
        assert abs(rb["n_evals"] - ra["n_evals"]) <= 1
    assert rel(b[1], a[1]) < 1e-6 and b[2] == pytest.approx(a[2], rel=1e-6)
