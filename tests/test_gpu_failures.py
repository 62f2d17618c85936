"""Failure paths through the C ABI, every one injected on the host.

The reference stops the program on a NaN after a forward FFT
(fftwfunction.f90:78-89) and ends a B solve on the mnbrak flags
(optimization.f90:271-292, 685-688) and on tau > TAU_MAX (310-314).  Here
each becomes the status code of the call, and the context stays usable for
the next field.  Nothing here faults or stalls the GPU: the bad values are
ordinary floating-point NaN/Inf in host arrays or parameters.
"""
import numpy as np
import pytest

import maxlq_b200 as mlq
from oracle.oracle import Oracle
from oracle.seedfield import seed_field

pytestmark = pytest.mark.gpu

N, Q = 16, 4.0


def good_field(seed=0, B=1.0):
    o = Oracle(N, Q, B)
    return o, o.rescale(o.divavg_free(seed_field(N, seed, 2.0, 2.0)))


def poisoned(u, value):
    v = u.copy()
    v[1, 3, 5, 7] = value
    return v


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_input_is_MLQ_ERR_NAN_and_the_context_recovers(precision, bad):
    o, u = good_field()
    c = mlq.MaxLq(N, Q, 1.0, precision=precision)
    v = poisoned(u, bad)
    for call in (c.calc_global_dLqdt_inclParts, c.eval_J, c.GradL2ForLq, c.state_load):
        with pytest.raises(mlq.MlqError) as e:
            call(v)
        assert e.value.status == mlq.MLQ_ERR_NAN, call.__name__
    # the flag was cleared: the same context evaluates a good field
    R = c.calc_global_dLqdt_inclParts(u)
    tol = 1e-10 if precision == "fp64" else 2e-5
    assert R[0] == pytest.approx(o.R_parts(u)[0], rel=tol)
    c.close()


def test_maxdlqdt_on_a_nan_field_returns_MLQ_ERR_NAN():
    _, u = good_field()
    c = mlq.MaxLq(N, Q, 1.0, max_iter=3)
    with pytest.raises(mlq.MlqError) as e:
        c.maxdLqdt(poisoned(u, np.nan))
    assert e.value.status == mlq.MLQ_ERR_NAN
    c.close()


def test_nan_arising_inside_the_loop_ends_it_with_MLQ_ERR_NAN():
    # constraintB = NaN between continuation steps: the retraction makes the
    # state NaN and the next forward transform reports it
    _, u = good_field()
    c = mlq.MaxLq(N, Q, 1.0, optim_tol=1e-14)
    c.state_load(u)
    it, st, _ = c.state_iterate(1)
    assert (it, st) == (1, mlq.MLQ_OK)
    c.set_B(float("nan"))
    with pytest.raises(mlq.MlqError) as e:
        c.state_iterate(2)
    assert e.value.status == mlq.MLQ_ERR_NAN
    c.close()


def test_fftfwd_nan_scan():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((N, N, N)) + 0j
    a[2, 2, 2] = np.nan
    c = mlq.MaxLq(N, Q, 1.0)
    with pytest.raises(mlq.MlqError) as e:
        c.fftfwd(a)
    assert e.value.status == mlq.MLQ_ERR_NAN
    with pytest.raises(mlq.MlqError) as e:
        c.fftfwdV(np.stack([a, a, a]))
    assert e.value.status == mlq.MLQ_ERR_NAN
    # fftbwd has no scan in the reference (98-113)
    out = c.fftbwd(a)
    assert np.isnan(out.real).any()
    c.close()


def test_mnbrak_flag_1_when_the_bracket_cannot_start():
    # tB0 = 0: tB = MACH_EPSILON, the shrink loop cannot run and myflag = 1
    # (optimization.f90:664, 677-688), as after a tau > TAU_MAX step
    o, u = good_field(2)
    d = o.divavg_free(o.hilbert_gradient(o.grad_l2(u), 1.5 - 1 / Q))
    c = mlq.MaxLq(N, Q, 1.0)
    _, fl_o = o.mnbrak(u, d, 0.0, 0.0)
    _, fl_c = c.mnbrak(u, d, 0.0, 0.0)
    assert fl_o == fl_c == 1
    c.close()


def test_mnbrak_along_an_ascent_direction_shrinks_to_rounding_like_the_oracle():
    # the negated descent direction: F(tau) = -R(retract(u + tau d)) rises, so
    # the shrink loop runs until tau is at the rounding level of R
    o, u = good_field(2)
    d = o.divavg_free(o.hilbert_gradient(o.grad_l2(u), 1.5 - 1 / Q))
    d = -d * np.sqrt(o.field_inner(u, u, "H") / o.field_inner(d, d, "H"))
    c = mlq.MaxLq(N, Q, 1.0)
    tb_o, fl_o = o.mnbrak(u, d, 0.0, 100.0)
    tb_c, fl_c = c.mnbrak(u, d, 0.0, 100.0)
    assert tb_o[1] < 1e-13 and tb_c[1] < 1e-13
    assert fl_c in (0, 1) and fl_o in (0, 1)
    c.close()


def test_tau_beyond_TAU_MAX_ends_the_loop():
    # normalizeGradient = .false. at a small B: the unscaled gradient is about
    # B^2 times u, so the first line minimum lies near tau = 1e3 > TAU_MAX
    B = 1e-3
    _, u = good_field(0, B)
    c = mlq.MaxLq(N, Q, B, normalize_gradient=0, optim_tol=1e-14, max_iter=5)
    _, it, st, rec = c.maxdLqdt(u)
    assert st == mlq.MLQ_ERR_TAU_MAX
    assert it == 1 and rec[-1]["tau"] == 0.0  # tau1 = 0 (313)
    c.close()
