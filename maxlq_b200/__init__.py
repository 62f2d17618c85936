"""maxlq_b200 -- B200 (sm_100a) engine for maxLq's Riemannian CG search.

Python mirror of the reference's subroutine surface (uniFabiB/maxLq,
optimization.f90, function_ops.f90, fftwfunction.f90) over the C ABI of
libmaxlq_b200.so.  Field arrays use the reference's memory layout: a vector
field is float64 of shape (3, N, N, N) indexed [c, z, y, x], i.e. the bytes of
the Fortran array U(1:n1, 1:n2, 1:n3, 1:3); a scalar field is (N, N, N).

    ctx = MaxLq(n=64, q=4.0, B=1.0)          # init_fft + module globals
    u = ctx.seed_field(seed=0, slope=2, k0=4)
    J = ctx.eval_J(u, "maxdLqdt")              # R(u)
    g = ctx.GradL2ForLq(u)
    u, iters, status, log = ctx.maxdLqdt(u)    # the CG loop for the current B
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import (  # noqa: F401
    ITER_CB, MLQ_ERR_BADARG, MLQ_ERR_IO, MLQ_ERR_J_DECREASED, MLQ_ERR_MNBRAK_ITMAX, MLQ_ERR_MNBRAK_UPHILL,
    MLQ_ERR_NAN, MLQ_ERR_NOT_BANDLIMITED,
    MLQ_ERR_TAU_MAX, MLQ_OK, MLQ_PREC_FP64, MLQ_PREC_MIXED, STATUS_NAMES, MlqIterInfo, MlqParams, dptr,
    load_library,
)

__all__ = ["MaxLq", "MlqError", "default_params", "band_cut", "seed_spectrum", "load_library", "ncdf_write_field",
           "ncdf_read_field"]

_MODES = {"maxdLqdt": 0, "LineMin": 1, "||u||_q": 2}
_INNER = {"L2": 0, "H_l^(3/2-1/q)": 1, "H": 1}
_LOOP_STOPS = (MLQ_ERR_MNBRAK_UPHILL, MLQ_ERR_MNBRAK_ITMAX, MLQ_ERR_TAU_MAX, MLQ_ERR_J_DECREASED)


class MlqError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status} {STATUS_NAMES.get(status, '?')}] {message}")
        self.status = status


def default_params(n: int, q: float, B: float = 1.0, **overrides) -> MlqParams:
    lib = load_library()
    p = MlqParams()
    lib.mlq_default_params(C.byref(p), n, q, B)
    for k, v in overrides.items():
        if k == "precision" and isinstance(v, str):
            v = {"fp64": MLQ_PREC_FP64, "mixed": MLQ_PREC_MIXED}[v]
        setattr(p, k, v)
    return p


def band_cut(n: int, order: float = 2.0) -> int:
    """Largest |j| a dealias of this order keeps (function_ops.f90:3374-3391)."""
    return load_library().mlq_band_cut(n, order)


def seed_spectrum(n: int, seed: int, slope: float, k0: float):
    """Host-only seeded spectrum (pruned half spectrum, see include/maxlq.h)."""
    lib = load_library()
    c = band_cut(n)
    nb, nx = 2 * c + 1, c + 1
    out = np.zeros((3, nb, nb, nx, 2))
    cut = C.c_int(0)
    st = lib.mlq_seed_spectrum(n, seed, slope, k0, dptr(out), C.byref(cut))
    if st != MLQ_OK:
        raise MlqError(st, "mlq_seed_spectrum")
    return out[..., 0] + 1j * out[..., 1], cut.value


def ncdf_write_field(path: str, u: np.ndarray, names=("Ux", "Uy", "Uz")) -> None:
    """save_field_R3toR3_ncdf (data_ops.f90:362-487): u of shape (3, n3, n2, n1)
    (the Fortran array U(1:n1, 1:n2, 1:n3, 1:3)) into a netCDF-3 classic file
    with dimensions x, y and an unlimited z, as the reference writes it."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.ndim != 4 or u.shape[0] != 3:
        raise ValueError("ncdf_write_field needs a (3, n3, n2, n1) field")
    _, n3, n2, n1 = u.shape
    st = load_library().mlq_ncdf_write_field(str(path).encode(), n1, n2, n3, dptr(u), *(x.encode() for x in names))
    if st != MLQ_OK:
        raise MlqError(st, f"ncdf_write_field {path}")


def ncdf_read_field(path: str, names=("Ux", "Uy", "Uz")) -> np.ndarray:
    """read_field_R3toR3_ncdf (data_ops.f90:1198-1397): the three named
    variables of a netCDF-3 file as a (3, n3, n2, n1) float64 field."""
    lib = load_library()
    dims = (C.c_int * 3)()
    st = lib.mlq_ncdf_read_dims(str(path).encode(), dims)
    if st != MLQ_OK:
        raise MlqError(st, f"ncdf_read_dims {path}")
    n1, n2, n3 = dims[0], dims[1], dims[2]
    u = np.empty((3, n3, n2, n1))
    st = lib.mlq_ncdf_read_field(str(path).encode(), n1, n2, n3, dptr(u), *(x.encode() for x in names))
    if st != MLQ_OK:
        raise MlqError(st, f"ncdf_read_field {path}")
    return u


class MaxLq:
    """One GPU context: the drop-in for the reference's hot-path modules."""

    def __init__(self, n: int, q: float, B: float = 1.0, precision: str | int = "fp64", **params):
        self._lib = load_library()
        self.params = default_params(n, q, B, precision=precision, **params)
        self.n, self.q, self.B = n, float(q), float(B)
        ctx = C.c_void_p()
        st = self._lib.mlq_init(C.byref(ctx), C.byref(self.params))
        if st != MLQ_OK:
            raise MlqError(st, "mlq_init failed (see stderr)")
        self._ctx = ctx

    # -- housekeeping ----------------------------------------------------------
    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.mlq_finalize(self._ctx)
            self._ctx = None

    fft_deallocate = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, what: str):
        if st != MLQ_OK:
            msg = self._lib.mlq_last_error(self._ctx)
            raise MlqError(st, f"{what}: {msg.decode() if msg else ''}")

    def _vec(self, u) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (3, self.n, self.n, self.n):
            raise ValueError(f"vector field must be (3,{self.n},{self.n},{self.n}), got {u.shape}")
        return u

    def _sca(self, f) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != (self.n,) * 3:
            raise ValueError(f"scalar field must be ({self.n},)*3, got {f.shape}")
        return f

    @property
    def kernel_launches(self) -> int:
        return self._lib.mlq_kernel_launches(self._ctx)

    @property
    def device_bytes(self) -> int:
        return self._lib.mlq_device_bytes(self._ctx)

    def set_B(self, B: float):
        self._check(self._lib.mlq_set_B(self._ctx, B), "set_B")
        self.B = float(B)

    # -- fftwfunction.f90 --------------------------------------------------------
    def fftfwd(self, u):
        a = np.ascontiguousarray(u, dtype=np.complex128)
        out = np.empty_like(a)
        self._check(self._lib.mlq_fft_fwd(self._ctx, dptr(a.view(np.float64)), dptr(out.view(np.float64))),
                    "fftfwd")
        return out

    def fftbwd(self, fu):
        a = np.ascontiguousarray(fu, dtype=np.complex128)
        out = np.empty_like(a)
        self._check(self._lib.mlq_fft_bwd(self._ctx, dptr(a.view(np.float64)), dptr(out.view(np.float64))),
                    "fftbwd")
        return out

    def fftfwdV(self, u):
        a = np.ascontiguousarray(u, dtype=np.complex128)
        out = np.empty_like(a)
        self._check(self._lib.mlq_fft_fwdV(self._ctx, dptr(a.view(np.float64)), dptr(out.view(np.float64))),
                    "fftfwdV")
        return out

    def fftbwdV(self, fu):
        a = np.ascontiguousarray(fu, dtype=np.complex128)
        out = np.empty_like(a)
        self._check(self._lib.mlq_fft_bwdV(self._ctx, dptr(a.view(np.float64)), dptr(out.view(np.float64))),
                    "fftbwdV")
        return out

    def fftfwdr(self, u):
        u = self._sca(u)
        out = np.empty((self.n, self.n, self.n // 2 + 1), dtype=np.complex128)
        self._check(self._lib.mlq_fft_fwdr(self._ctx, dptr(u), dptr(out.view(np.float64))), "fftfwdr")
        return out

    def fftbwdr(self, fu):
        a = np.ascontiguousarray(fu, dtype=np.complex128)
        out = np.empty((self.n,) * 3)
        self._check(self._lib.mlq_fft_bwdr(self._ctx, dptr(a.view(np.float64)), dptr(out)), "fftbwdr")
        return out

    # -- function_ops.f90 ----------------------------------------------------------
    def dealias_scalar(self, g, order: float):
        g = self._sca(g).copy()
        self._check(self._lib.mlq_dealias_scalar(self._ctx, dptr(g), order), "dealias_scalar")
        return g

    def gradient(self, f):
        f = self._sca(f)
        out = np.empty((3,) + f.shape)
        self._check(self._lib.mlq_gradient(self._ctx, dptr(f), dptr(out)), "gradient")
        return out

    def divergence(self, u):
        u = self._vec(u)
        out = np.empty(u.shape[1:])
        self._check(self._lib.mlq_divergence(self._ctx, dptr(u), dptr(out)), "divergence")
        return out

    def laplacian(self, u):
        u = self._vec(u).copy()
        self._check(self._lib.mlq_laplacian(self._ctx, dptr(u)), "laplacian")
        return u

    def solve_poisson(self, f, l: float = 1.0):
        f = self._sca(f)
        out = np.empty_like(f)
        self._check(self._lib.mlq_solve_poisson(self._ctx, dptr(f), l, dptr(out)), "solve_poisson")
        return out

    def calc_uk(self, u, k: float):
        u = self._vec(u)
        out = np.empty(u.shape[1:])
        self._check(self._lib.mlq_calc_uk(self._ctx, dptr(u), k, dptr(out)), "calc_uk")
        return out

    def divAvg_free(self, u):
        u = self._vec(u).copy()
        self._check(self._lib.mlq_divavg_free(self._ctx, dptr(u)), "divAvg_free")
        return u

    def HilbertGradient(self, grad, order: float):
        g = self._vec(grad).copy()
        self._check(self._lib.mlq_hilbert_gradient(self._ctx, dptr(g), order), "HilbertGradient")
        return g

    def global_summed_field_inner_product(self, f, g, mytype: str = "L2") -> float:
        out = C.c_double(0.0)
        st = self._lib.mlq_inner_product(self._ctx, dptr(self._vec(f)), dptr(self._vec(g)), _INNER[mytype],
                                         C.byref(out))
        self._check(st, "inner_product")
        return out.value

    def calc0thFourierModes(self, u):
        out = np.zeros(3)
        self._check(self._lib.mlq_zeroth_modes(self._ctx, dptr(self._vec(u)), dptr(out)), "calc0thFourierModes")
        return out

    def calc_global_Lq_norm(self, u) -> float:
        out = C.c_double(0.0)
        self._check(self._lib.mlq_lq_norm(self._ctx, dptr(self._vec(u)), C.byref(out)), "calc_global_Lq_norm")
        return out.value

    def rescaleLqNorm(self, u, B: float | None = None):
        u = self._vec(u).copy()
        self._check(self._lib.mlq_rescale(self._ctx, dptr(u), self.B if B is None else B), "rescaleLqNorm")
        return u

    def calcConstraintDerivativeL2(self, u):
        u = self._vec(u)
        out = np.empty_like(u)
        self._check(self._lib.mlq_normal_l2(self._ctx, dptr(u), dptr(out)), "calcConstraintDerivativeL2")
        return out

    def vectorTransport(self, u, q, B, eta, xi):
        u, eta, xi = self._vec(u), self._vec(eta), self._vec(xi)
        out = np.empty_like(u)
        st = self._lib.mlq_vector_transport(self._ctx, dptr(u), q, B, dptr(eta), dptr(xi), dptr(out))
        self._check(st, "vectorTransport")
        return out

    def calc_global_dLqdt_inclParts(self, u) -> np.ndarray:
        out = np.zeros(3)
        self._check(self._lib.mlq_R_parts(self._ctx, dptr(self._vec(u)), dptr(out)), "calc_global_dLqdt_inclParts")
        return out

    def GradL2ForLq(self, u):
        u = self._vec(u)
        out = np.empty_like(u)
        self._check(self._lib.mlq_grad_l2(self._ctx, dptr(u), dptr(out)), "GradL2ForLq")
        return out

    # -- optimization.f90 -----------------------------------------------------------
    def eval_J(self, u, mysystem: str = "maxdLqdt") -> float:
        out = C.c_double(0.0)
        self._check(self._lib.mlq_eval_J(self._ctx, dptr(self._vec(u)), _MODES[mysystem], C.byref(out)), "eval_J")
        return out.value

    def kappa_test(self, phi, gradJ, phi_pert, mysystem: str = "maxdLqdt", inner_product_space: str = "L2",
                   n: int = 16) -> dict:
        """kappa_test (optimization.f90:957-1129) with a given perturbation:
        J at phi and at phi + eps_i phi_pert (eps_i = 10^(-7 - n/2 + i)), the
        kappa table, the reference's best kappa and the adjusted kappa.  The
        perturbation must be band-limited like every field this engine takes
        (the reference's own perturbation files are not part of the path)."""
        lib = self._lib
        eps = np.empty(n)
        self._check(lib.mlq_kappa_epsilons(n, dptr(eps)), "kappa_epsilons")
        phi = self._vec(phi)
        pert = self._vec(phi_pert)
        inner = self.global_summed_field_inner_product(gradJ, pert, inner_product_space)
        J0 = self.eval_J(phi, mysystem)
        J1 = np.array([self.eval_J(phi + e * pert, mysystem) for e in eps])
        table = np.empty((n, 5))
        frac, best = C.c_double(0.0), C.c_double(0.0)
        bi = C.c_int(0)
        self._check(lib.mlq_kappa_table(J0, dptr(J1), inner, n, dptr(table), C.byref(frac), C.byref(bi),
                                        C.byref(best)), "kappa_table")
        return {"epsilon": table[:, 0], "inner_product": inner, "deltaJ": table[:, 2], "kappa": table[:, 3],
                "kappa_adjusted": table[:, 4], "adjust_factor": frac.value, "best_index": bi.value,
                "best_kappa": best.value, "J0": J0}

    # -- diagnostics (maxdLpdt.f90:263-299, optimization.f90:119-123, 377-384) --
    def calculate_spectral_data(self, u=None, normalize: bool = True):
        """(kk_max, spectrum) of u, or of the resident state when u is None."""
        out = np.zeros(2 * self.n)
        if u is None:
            self._check(self._lib.mlq_state_spectral_data(self._ctx, 1 if normalize else 0, dptr(out)),
                        "state_spectral_data")
        else:
            self._check(self._lib.mlq_spectral_data(self._ctx, dptr(self._vec(u)), 1 if normalize else 0, dptr(out)),
                        "spectral_data")
        return out[: self.n].copy(), out[self.n:].copy()

    def calc_global_summed_enstrophy(self, u) -> float:
        out = C.c_double(0.0)
        self._check(self._lib.mlq_summed_enstrophy(self._ctx, dptr(self._vec(u)), C.byref(out)), "summed_enstrophy")
        return out.value

    def calc_global_dEnstrophydt(self, u) -> np.ndarray:
        out = np.zeros(3)
        self._check(self._lib.mlq_dEnstrophydt(self._ctx, dptr(self._vec(u)), dptr(out)), "dEnstrophydt")
        return out

    def calc_local_pointwise_dLqdt_inclParts(self, u) -> np.ndarray:
        out = np.zeros((3, self.n, self.n, self.n))
        self._check(self._lib.mlq_pointwise_R(self._ctx, dptr(self._vec(u)), dptr(out)), "pointwise_R")
        return out

    def kappa_test_pert(self, mytype: str, m1: float = 0.0, m2: float = 0.0, m3: float = 0.0, loaded=None,
                        seed: int = 0):
        """kappa_test_pert (function_ops.f90:615-977): (phi_pert, successful).
        loaded: the field a load-* type reads from its file (None: no file,
        phi formed from zeros and successful False)."""
        out = np.zeros((3, self.n, self.n, self.n))
        src = None if loaded is None else dptr(self._vec(loaded))
        st = self._lib.mlq_kappa_perturbation(self._ctx, mytype.encode(), m1, m2, m3, src, seed, dptr(out))
        if st == MLQ_ERR_IO:
            return out, False
        self._check(st, "kappa_test_pert")
        return out, True

    def mnbrak(self, phi, grad, tA0: float, tB0: float):
        """Returns (tau_brack, myflag) like the Fortran function and its inout flag."""
        tb = np.zeros(2)
        flag = C.c_int(0)
        st = self._lib.mlq_mnbrak(self._ctx, dptr(self._vec(phi)), dptr(self._vec(grad)), tA0, tB0, dptr(tb),
                                  C.byref(flag))
        self._check(st, "mnbrak")
        return tb, flag.value

    def brent(self, phi, grad, tau_brack) -> float:
        tb = np.ascontiguousarray(tau_brack, dtype=np.float64)
        out = C.c_double(0.0)
        st = self._lib.mlq_brent(self._ctx, dptr(self._vec(phi)), dptr(self._vec(grad)), dptr(tb), C.byref(out))
        self._check(st, "brent")
        return out.value

    def _runner(self, callback):
        records = []

        def _cb(info_p, _user):
            rec = info_p.contents.as_dict()
            records.append(rec)
            if callback is not None:
                callback(rec)

        return records, ITER_CB(_cb)

    def maxdLqdt(self, u, start_iter: int = 0, callback=None):
        """optimization.f90:7-514 on a copy of u; returns (u, iter, status, records).

        status is MLQ_OK or the loop-ending code (mnbrak flags, tau > TAU_MAX,
        J decreasing), which the reference reports through messages and flags.
        """
        u = self._vec(u).copy()
        records, cb = self._runner(callback)
        it = C.c_int(0)
        st = self._lib.mlq_maxdlqdt(self._ctx, dptr(u), start_iter, cb, None, C.byref(it))
        if st not in (MLQ_OK,) + _LOOP_STOPS:
            self._check(st, "maxdLqdt")
        return u, it.value, st, records

    # -- device-resident state ------------------------------------------------------
    def state_load(self, u):
        self._check(self._lib.mlq_state_load(self._ctx, dptr(self._vec(u))), "state_load")

    def state_store(self):
        u = np.empty((3, self.n, self.n, self.n))
        self._check(self._lib.mlq_state_store(self._ctx, dptr(u)), "state_store")
        return u

    def state_iterate(self, n_iter: int, callback=None):
        records, cb = self._runner(callback)
        it = C.c_int(0)
        st = self._lib.mlq_state_iterate(self._ctx, n_iter, cb, None, C.byref(it))
        if st not in (MLQ_OK,) + _LOOP_STOPS:
            self._check(st, "state_iterate")
        return it.value, st, records

    def state_R(self):
        out = np.zeros(3)
        nrm = C.c_double(0.0)
        self._check(self._lib.mlq_state_R(self._ctx, dptr(out), C.byref(nrm)), "state_R")
        return out, nrm.value

    def state_step(self, u, callback=None):
        """One CG iteration on a host field (H2D, iterate, D2H); u updated in place."""
        if not (isinstance(u, np.ndarray) and u.dtype == np.float64 and u.flags.c_contiguous
                and u.shape == (3, self.n, self.n, self.n)):
            raise ValueError("state_step needs a C-contiguous float64 (3,N,N,N) array")
        records, cb = self._runner(callback)
        st = self._lib.mlq_state_step(self._ctx, dptr(u), cb, None)
        if st not in (MLQ_OK,) + _LOOP_STOPS:
            self._check(st, "state_step")
        return st, records

    def profile(self, on: bool | int = True):
        """Per-kernel device timing; on=2 also keys x-stage launches by functor."""
        level = int(on) if not isinstance(on, bool) else (1 if on else 0)
        self._check(self._lib.mlq_profile_enable(self._ctx, level), "profile_enable")

    def profile_report(self, reset: bool = True) -> dict:
        import json
        need = self._lib.mlq_profile_report(self._ctx, None, 0, 0)
        if need < 0:
            self._check(-need, "profile_report")
        buf = C.create_string_buffer(need + 16)
        self._lib.mlq_profile_report(self._ctx, buf, need + 16, 1 if reset else 0)
        return {k: {"launches": v[0], "ms": v[1], "bytes": v[2]} for k, v in json.loads(buf.value.decode()).items()}

    def kernel_config(self) -> dict:
        """Pass-kernel family, precision and the autotuned y/z tile shapes."""
        import json
        need = self._lib.mlq_kernel_config(self._ctx, None, 0)
        if need < 0:
            self._check(-need, "kernel_config")
        buf = C.create_string_buffer(need + 16)
        self._lib.mlq_kernel_config(self._ctx, buf, need + 16)
        return json.loads(buf.value.decode())

    def seed_field(self, seed: int = 0, slope: float = 2.0, k0: float = 4.0):
        u = np.empty((3, self.n, self.n, self.n))
        self._check(self._lib.mlq_seed_field(self._ctx, seed, slope, k0, dptr(u)), "seed_field")
        return u
