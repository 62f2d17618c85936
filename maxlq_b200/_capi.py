"""ctypes binding of libmaxlq_b200.so (the C ABI declared in include/maxlq.h).

The library is required: importing this module without it raises, there is no
CPU fallback.  Build it with ``python -m maxlq_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmaxlq_b200.so")

MLQ_OK = 0
MLQ_ERR_NAN = 1
MLQ_ERR_MNBRAK_UPHILL = 2
MLQ_ERR_MNBRAK_ITMAX = 3
MLQ_ERR_TAU_MAX = 4
MLQ_ERR_J_DECREASED = 5
MLQ_ERR_TIMEOUT = 6
MLQ_ERR_OOM = 7
MLQ_ERR_BADARG = 8
MLQ_ERR_CUDA = 9
MLQ_ERR_NOT_BANDLIMITED = 10
MLQ_ERR_IO = 11

MLQ_PREC_FP64 = 0
MLQ_PREC_MIXED = 1

STATUS_NAMES = {
    0: "ok", 1: "nan", 2: "mnbrak uphill", 3: "mnbrak itmax", 4: "tau > TAU_MAX", 5: "J decreased",
    6: "device timeout", 7: "out of device memory", 8: "bad argument", 9: "cuda error", 10: "not band-limited",
    11: "file error",
}


class MlqParams(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("q", C.c_double), ("B", C.c_double), ("visc", C.c_double), ("lambda1", C.c_double),
        ("visc_coef", C.c_double), ("press_coef", C.c_double), ("to_dealias", C.c_int),
        ("use_e_u_auto", C.c_int), ("use_e_u", C.c_int), ("dealias_e_u", C.c_int),
        ("use_tangential_gradient", C.c_int), ("use_conjugate_gradient", C.c_int),
        ("use_riemannian_geometry", C.c_int), ("normalize_gradient", C.c_int),
        ("reset_momentum_every", C.c_int), ("rolling_size", C.c_int), ("max_iter", C.c_int),
        ("optim_tol", C.c_double), ("precision", C.c_int), ("device", C.c_int),
    ]


class MlqIterInfo(C.Structure):
    _fields_ = [
        ("iter", C.c_int),
        ("tau_a", C.c_double), ("tau", C.c_double), ("tau_b", C.c_double),
        ("J0", C.c_double), ("deltaJ", C.c_double), ("J1", C.c_double),
        ("beta", C.c_double), ("alpha", C.c_double),
        ("norm_grad", C.c_double), ("norm_td0", C.c_double), ("norm_d1", C.c_double),
        ("u_norm_q", C.c_double),
        ("R", C.c_double), ("R12", C.c_double), ("R3", C.c_double),
        ("ortho_check", C.c_double), ("div_check", C.c_double),
        ("mean_d1", C.c_double * 3), ("mean_u", C.c_double * 3),
        ("n_evals", C.c_int), ("mnbrak_flag", C.c_int), ("status", C.c_int),
        ("seconds", C.c_double),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if isinstance(v, C.Array) else v
        return d


ITER_CB = C.CFUNCTYPE(None, C.POINTER(MlqIterInfo), C.c_void_p)
_DP = C.POINTER(C.c_double)
_VP = C.c_void_p

# name -> (restype, argtypes); exactly the entry points of include/maxlq.h
SIGNATURES = {
    "mlq_default_params": (None, [C.POINTER(MlqParams), C.c_int, C.c_double, C.c_double]),
    "mlq_init": (C.c_int, [C.POINTER(_VP), C.POINTER(MlqParams)]),
    "mlq_finalize": (C.c_int, [_VP]),
    "mlq_last_error": (C.c_char_p, [_VP]),
    "mlq_set_B": (C.c_int, [_VP, C.c_double]),
    "mlq_kernel_launches": (C.c_longlong, [_VP]),
    "mlq_device_bytes": (C.c_longlong, [_VP]),
    "mlq_fft_fwd": (C.c_int, [_VP, _DP, _DP]),
    "mlq_fft_bwd": (C.c_int, [_VP, _DP, _DP]),
    "mlq_fft_fwdV": (C.c_int, [_VP, _DP, _DP]),
    "mlq_spectral_data": (C.c_int, [_VP, _DP, C.c_int, _DP]),
    "mlq_state_spectral_data": (C.c_int, [_VP, C.c_int, _DP]),
    "mlq_summed_enstrophy": (C.c_int, [_VP, _DP, _DP]),
    "mlq_dEnstrophydt": (C.c_int, [_VP, _DP, _DP]),
    "mlq_pointwise_R": (C.c_int, [_VP, _DP, _DP]),
    "mlq_kappa_perturbation": (C.c_int, [_VP, C.c_char_p, C.c_double, C.c_double, C.c_double, _DP, C.c_ulonglong,
                                         _DP]),
    "mlq_fft_bwdV": (C.c_int, [_VP, _DP, _DP]),
    "mlq_fft_fwdr": (C.c_int, [_VP, _DP, _DP]),
    "mlq_fft_bwdr": (C.c_int, [_VP, _DP, _DP]),
    "mlq_dealias_scalar": (C.c_int, [_VP, _DP, C.c_double]),
    "mlq_gradient": (C.c_int, [_VP, _DP, _DP]),
    "mlq_divergence": (C.c_int, [_VP, _DP, _DP]),
    "mlq_laplacian": (C.c_int, [_VP, _DP]),
    "mlq_solve_poisson": (C.c_int, [_VP, _DP, C.c_double, _DP]),
    "mlq_calc_uk": (C.c_int, [_VP, _DP, C.c_double, _DP]),
    "mlq_divavg_free": (C.c_int, [_VP, _DP]),
    "mlq_hilbert_gradient": (C.c_int, [_VP, _DP, C.c_double]),
    "mlq_inner_product": (C.c_int, [_VP, _DP, _DP, C.c_int, _DP]),
    "mlq_zeroth_modes": (C.c_int, [_VP, _DP, _DP]),
    "mlq_lq_norm": (C.c_int, [_VP, _DP, _DP]),
    "mlq_rescale": (C.c_int, [_VP, _DP, C.c_double]),
    "mlq_normal_l2": (C.c_int, [_VP, _DP, _DP]),
    "mlq_vector_transport": (C.c_int, [_VP, _DP, C.c_double, C.c_double, _DP, _DP, _DP]),
    "mlq_R_parts": (C.c_int, [_VP, _DP, _DP]),
    "mlq_grad_l2": (C.c_int, [_VP, _DP, _DP]),
    "mlq_eval_J": (C.c_int, [_VP, _DP, C.c_int, _DP]),
    "mlq_mnbrak": (C.c_int, [_VP, _DP, _DP, C.c_double, C.c_double, _DP, C.POINTER(C.c_int)]),
    "mlq_brent": (C.c_int, [_VP, _DP, _DP, _DP, _DP]),
    "mlq_maxdlqdt": (C.c_int, [_VP, _DP, C.c_int, ITER_CB, _VP, C.POINTER(C.c_int)]),
    "mlq_state_load": (C.c_int, [_VP, _DP]),
    "mlq_state_store": (C.c_int, [_VP, _DP]),
    "mlq_state_iterate": (C.c_int, [_VP, C.c_int, ITER_CB, _VP, C.POINTER(C.c_int)]),
    "mlq_state_R": (C.c_int, [_VP, _DP, _DP]),
    "mlq_state_step": (C.c_int, [_VP, _DP, ITER_CB, _VP]),
    "mlq_profile_enable": (C.c_int, [_VP, C.c_int]),
    "mlq_profile_report": (C.c_int, [_VP, C.c_char_p, C.c_int, C.c_int]),
    "mlq_kernel_config": (C.c_int, [_VP, C.c_char_p, C.c_int]),
    "mlq_seed_field": (C.c_int, [_VP, C.c_ulonglong, C.c_double, C.c_double, _DP]),
    "mlq_seed_spectrum": (C.c_int, [C.c_int, C.c_ulonglong, C.c_double, C.c_double, _DP, C.POINTER(C.c_int)]),
    "mlq_band_cut": (C.c_int, [C.c_int, C.c_double]),
    "mlq_dealias_scalar_noalloc": (C.c_int, [_DP, C.c_int, C.c_double]),
    "mlq_kappa_epsilons": (C.c_int, [C.c_int, _DP]),
    "mlq_kappa_table": (C.c_int, [C.c_double, _DP, C.c_double, C.c_int, _DP, _DP, C.POINTER(C.c_int), _DP]),
    "mlq_ncdf_write_field": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _DP, C.c_char_p, C.c_char_p,
                                       C.c_char_p]),
    "mlq_ncdf_read_dims": (C.c_int, [C.c_char_p, C.POINTER(C.c_int)]),
    "mlq_ncdf_read_field": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _DP, C.c_char_p, C.c_char_p,
                                      C.c_char_p]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m maxlq_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_DP)
