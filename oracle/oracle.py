"""ctypes wrapper around the CPU oracle (oracle/mlq_oracle.cpp).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm import this module as the checker.  The product
package (maxlq_b200) never imports it.

Parity unpinned: no golden vectors exist in the reference and its Fortran
build is unavailable here; see mlq_oracle.h for how the oracle is checked.

Fields are numpy float64 arrays shaped (3, N, N, N) indexed [c, z, y, x]:
byte-for-byte the reference's Fortran array Uvec(1:n1, 1:n2, 1:n3, 1:3)
(column-major, x fastest).  Scalars are (N, N, N).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -fopenmp) into oracle/_build."""
    src = os.path.join(_HERE, "mlq_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcParams(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("q", C.c_double), ("B", C.c_double), ("visc", C.c_double),
        ("lambda1", C.c_double), ("visc_coef", C.c_double), ("press_coef", C.c_double),
        ("to_dealias", C.c_int), ("use_e_u", C.c_int), ("dealias_e_u", C.c_int), ("threads", C.c_int),
    ]


class OrcIterInfo(C.Structure):
    _fields_ = [
        ("iter", C.c_int),
        ("tau_a", C.c_double), ("tau", C.c_double), ("tau_b", C.c_double),
        ("J0", C.c_double), ("deltaJ", C.c_double), ("J1", C.c_double),
        ("beta", C.c_double), ("alpha", C.c_double),
        ("norm_grad", C.c_double), ("norm_td0", C.c_double), ("norm_d1", C.c_double),
        ("u_norm_q", C.c_double),
        ("R", C.c_double), ("R12", C.c_double), ("R3", C.c_double),
        ("n_evals", C.c_int), ("mnbrak_flag", C.c_int),
    ]


ITER_CB = C.CFUNCTYPE(None, C.POINTER(OrcIterInfo), C.c_void_p)
_DP = C.POINTER(C.c_double)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    sig = {
        "orc_default_params": (None, [C.POINTER(OrcParams), C.c_int, C.c_double, C.c_double]),
        "orc_create": (vp, [C.POINTER(OrcParams)]),
        "orc_destroy": (None, [vp]),
        "orc_eval_count": (C.c_int, [vp]),
        "orc_fft_c2c": (None, [vp, _DP, C.c_int]),
        "orc_dealias_scalar": (None, [vp, _DP, C.c_double]),
        "orc_spectral_data": (None, [vp, _DP, _DP, C.c_int]),
        "orc_summed_enstrophy": (C.c_double, [vp, _DP]),
        "orc_dEnstrophydt": (None, [vp, _DP, _DP]),
        "orc_pointwise_R": (None, [vp, _DP, _DP]),
        "orc_kappa_pert": (C.c_int, [vp, C.c_char_p, C.c_double, C.c_double, C.c_double, _DP, C.c_ulonglong,
                                     _DP]),
        "orc_gradient": (None, [vp, _DP, _DP]),
        "orc_divergence": (None, [vp, _DP, _DP]),
        "orc_laplacian": (None, [vp, _DP]),
        "orc_solve_poisson": (None, [vp, _DP, C.c_double, _DP]),
        "orc_calc_uk": (None, [vp, _DP, C.c_double, _DP]),
        "orc_unit_vector": (None, [vp, _DP, _DP]),
        "orc_divavg_free": (None, [vp, _DP]),
        "orc_hilbert_gradient": (None, [vp, _DP, C.c_double]),
        "orc_inner_product": (C.c_double, [vp, _DP, _DP, C.c_int]),
        "orc_field_inner": (C.c_double, [vp, _DP, _DP, C.c_int]),
        "orc_zeroth_modes": (None, [vp, _DP]),
        "orc_lq_norm": (C.c_double, [vp, _DP]),
        "orc_rescale": (None, [vp, _DP, C.c_double]),
        "orc_normal_l2": (None, [vp, _DP, _DP]),
        "orc_vector_transport": (None, [vp, _DP, C.c_double, C.c_double, _DP, _DP, _DP]),
        "orc_R_parts": (None, [vp, _DP, _DP]),
        "orc_grad_l2": (None, [vp, _DP, _DP]),
        "orc_eval_J": (C.c_double, [vp, _DP, C.c_int]),
        "orc_mnbrak": (C.c_int, [vp, _DP, _DP, C.c_double, C.c_double, _DP, C.POINTER(C.c_int)]),
        "orc_brent": (C.c_double, [vp, _DP, _DP, _DP]),
        "orc_maxdlqdt": (C.c_int, [vp, _DP, C.c_int, C.c_double, C.c_int, ITER_CB, vp, C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


MODE = {"maxdLqdt": 0, "LineMin": 1, "||u||_q": 2}


class Oracle:
    """One reference 'rank' holding the whole N^3 box (local_N = N)."""

    def __init__(self, n: int, q: float, B: float = 1.0, threads: int = 0, **overrides):
        lib = _load()
        p = OrcParams()
        lib.orc_default_params(C.byref(p), n, q, B)
        p.threads = threads
        for k, v in overrides.items():
            setattr(p, k, v)
        self.params = p
        self.n, self.q, self.B = n, q, B
        self._lib = lib
        self._ctx = lib.orc_create(C.byref(p))

    def close(self):
        if self._ctx:
            self._lib.orc_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers -----------------------------------------------------------
    def _vec(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == (3, self.n, self.n, self.n), u.shape
        return u

    def _sca(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        assert f.shape == (self.n,) * 3, f.shape
        return f

    @property
    def eval_count(self) -> int:
        return self._lib.orc_eval_count(self._ctx)

    # -- fftwfunction.f90 ---------------------------------------------------
    def fft_c2c(self, a: np.ndarray, direction: int) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.complex128).copy()
        self._lib.orc_fft_c2c(self._ctx, a.view(np.float64).ctypes.data_as(_DP), direction)
        return a

    # -- function_ops.f90 ---------------------------------------------------
    def dealias_scalar(self, g, order):
        g = self._sca(g).copy()
        self._lib.orc_dealias_scalar(self._ctx, _p(g), order)
        return g

    def gradient(self, f):
        f = self._sca(f)
        out = np.empty((3,) + f.shape)
        self._lib.orc_gradient(self._ctx, _p(f), _p(out))
        return out

    def divergence(self, u):
        u = self._vec(u)
        out = np.empty(u.shape[1:])
        self._lib.orc_divergence(self._ctx, _p(u), _p(out))
        return out

    def laplacian(self, u):
        u = self._vec(u).copy()
        self._lib.orc_laplacian(self._ctx, _p(u))
        return u

    def solve_poisson(self, f, l=1.0):
        f = self._sca(f)
        out = np.empty_like(f)
        self._lib.orc_solve_poisson(self._ctx, _p(f), l, _p(out))
        return out

    def calc_uk(self, u, k):
        u = self._vec(u)
        out = np.empty(u.shape[1:])
        self._lib.orc_calc_uk(self._ctx, _p(u), k, _p(out))
        return out

    def unit_vector(self, u):
        u = self._vec(u)
        out = np.empty_like(u)
        self._lib.orc_unit_vector(self._ctx, _p(u), _p(out))
        return out

    def divavg_free(self, u):
        u = self._vec(u).copy()
        self._lib.orc_divavg_free(self._ctx, _p(u))
        return u

    def hilbert_gradient(self, g, order):
        g = self._vec(g).copy()
        self._lib.orc_hilbert_gradient(self._ctx, _p(g), order)
        return g

    def inner_product(self, f, g, htype="L2"):
        return self._lib.orc_inner_product(self._ctx, _p(self._sca(f)), _p(self._sca(g)), int(htype != "L2"))

    def field_inner(self, f, g, htype="L2"):
        return self._lib.orc_field_inner(self._ctx, _p(self._vec(f)), _p(self._vec(g)), int(htype != "L2"))

    def zeroth_modes(self, u):
        out = np.empty(3)
        self._lib.orc_zeroth_modes(self._ctx, _p(self._vec(u)), _p(out))
        return out

    def lq_norm(self, u):
        return self._lib.orc_lq_norm(self._ctx, _p(self._vec(u)))

    def rescale(self, u, B=None):
        u = self._vec(u).copy()
        self._lib.orc_rescale(self._ctx, _p(u), self.B if B is None else B)
        return u

    def normal_l2(self, u):
        u = self._vec(u)
        out = np.empty_like(u)
        self._lib.orc_normal_l2(self._ctx, _p(u), _p(out))
        return out

    def vector_transport(self, u, eta, xi, q=None, B=None):
        u, eta, xi = self._vec(u), self._vec(eta), self._vec(xi)
        out = np.empty_like(u)
        self._lib.orc_vector_transport(self._ctx, _p(u), self.q if q is None else q,
                                       self.B if B is None else B, _p(eta), _p(xi), _p(out))
        return out

    def R_parts(self, u):
        out = np.empty(3)
        self._lib.orc_R_parts(self._ctx, _p(self._vec(u)), _p(out))
        return out

    def grad_l2(self, u):
        u = self._vec(u)
        out = np.empty_like(u)
        self._lib.orc_grad_l2(self._ctx, _p(u), _p(out))
        return out

    # -- optimization.f90 ---------------------------------------------------
    def eval_J(self, u, mode="maxdLqdt"):
        return self._lib.orc_eval_J(self._ctx, _p(self._vec(u)), MODE[mode])

    def mnbrak(self, phi, d, tA0, tB0):
        tb = np.zeros(2)
        flag = C.c_int(0)
        self._lib.orc_mnbrak(self._ctx, _p(self._vec(phi)), _p(self._vec(d)), tA0, tB0, _p(tb), C.byref(flag))
        return tb, flag.value

    def brent(self, phi, d, tau_brack):
        tb = np.ascontiguousarray(tau_brack, dtype=np.float64)
        return self._lib.orc_brent(self._ctx, _p(self._vec(phi)), _p(self._vec(d)), _p(tb))

    # -- diagnostics (maxdLpdt.f90:263-299, optimization.f90:119-123, 377-384) --
    def spectral_data(self, u, normalize=True):
        """calculate_spectral_data: (kk_max, spectrum), each of length n."""
        out = np.zeros(2 * self.n)
        self._lib.orc_spectral_data(self._ctx, _p(self._vec(u)), _p(out), 1 if normalize else 0)
        return out[: self.n].copy(), out[self.n:].copy()

    def summed_enstrophy(self, u):
        return self._lib.orc_summed_enstrophy(self._ctx, _p(self._vec(u)))

    def dEnstrophydt(self, u):
        out = np.zeros(3)
        self._lib.orc_dEnstrophydt(self._ctx, _p(self._vec(u)), _p(out))
        return out

    def pointwise_R(self, u):
        out = np.zeros((3, self.n, self.n, self.n))
        self._lib.orc_pointwise_R(self._ctx, _p(self._vec(u)), _p(out))
        return out

    def kappa_test_pert(self, mytype, m1=0.0, m2=0.0, m3=0.0, loaded=None, seed=0):
        """kappa_test_pert (function_ops.f90:615-977): (phi, successful).
        loaded: the field a load-* type reads from its file (None: no file)."""
        out = np.zeros((3, self.n, self.n, self.n))
        src = None if loaded is None else _p(self._vec(loaded))
        r = self._lib.orc_kappa_pert(self._ctx, mytype.encode(), m1, m2, m3, src, seed, _p(out))
        if r < 0:
            raise ValueError("unknown perturbation type " + mytype)
        return out, bool(r)

    def maxdlqdt(self, u, max_iter=99999, optim_tol=1e-5, start_iter=0, callback=None):
        """Run the CG loop on a copy of u; returns (u, iterations, flag, records)."""
        u = self._vec(u).copy()
        records = []

        def _cb(info_p, _user):
            i = info_p.contents
            rec = {name: getattr(i, name) for name, _ in OrcIterInfo._fields_}
            records.append(rec)
            if callback is not None:
                callback(rec)

        cb = ITER_CB(_cb)
        flag = C.c_int(0)
        it = self._lib.orc_maxdlqdt(self._ctx, _p(u), max_iter, optim_tol, start_iter, cb, None, C.byref(flag))
        return u, it, flag.value, records
