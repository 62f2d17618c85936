"""The C ABI library without a GPU: it loads, exports every declared symbol,
and its host-only pieces (band cut, seeded spectra) agree with the checker."""
import ctypes
import os
import re

import numpy as np
import pytest

import maxlq_b200
from maxlq_b200 import _capi
from oracle import seedfield

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "maxlq.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mlq_\w+)\s*\(", text)) - {"mlq_iter_cb"})


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 38
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert set(names) == set(_capi.SIGNATURES), set(names) ^ set(_capi.SIGNATURES)


def test_default_params_mirror_reference_globals():
    p = maxlq_b200.default_params(256, 4.0, 1.0)
    assert p.visc == 1.0 and p.lambda1 == 0.1            # global_variables.f90:8, 31
    assert p.reset_momentum_every == 25 and p.rolling_size == 10  # 35, 36
    assert p.max_iter == 99999 and p.optim_tol == 1e-5   # 26, initialize.f90:99
    assert maxlq_b200.default_params(1024, 4.0).optim_tol == 1e-4  # initialize.f90:97


@pytest.mark.parametrize("n", [8, 12, 16, 48, 64, 96, 128, 256, 512, 1024])
@pytest.mark.parametrize("order", [0.0, 1.0, 1.5, 2.0, 3.0])
def test_band_cut_matches_reference_expression(n, order):
    assert maxlq_b200.band_cut(n, order) == seedfield.band_cut(n, order)


def test_band_cut_values():
    # 2/3 rule: keep |j| <= N/3 (inclusive when N is divisible by 3)
    assert [maxlq_b200.band_cut(n) for n in (48, 64, 96, 512, 1024)] == [16, 21, 32, 170, 341]
    assert maxlq_b200.band_cut(64, 1.0) == 32  # order 1: nothing removed


@pytest.mark.parametrize("n,seed", [(16, 0), (48, 7), (64, 31)])
def test_seed_spectrum_matches_independent_generator(n, seed):
    a, ca = maxlq_b200.seed_spectrum(n, seed, 2.0, n / 16)
    b, cb = seedfield.seed_spectrum(n, seed, 2.0, n / 16)
    assert ca == cb
    assert np.abs(a - b).max() < 1e-14 * np.abs(b).max()


def test_philox_known_answers():
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, exp in kat:
        got = seedfield.philox4x32_10(np.array(ctr, dtype=np.uint32)[None], np.array(key, dtype=np.uint32))[0]
        assert tuple(int(x) for x in got) == exp


def test_seed_field_is_divfree_meanfree_dealiased():
    from oracle.ref_numpy import RefNumpy
    n = 16
    u = seedfield.seed_field(n, 2, 2.0, 4.0)
    r = RefNumpy(n, 4.0)
    assert np.abs(r.divergence(u)).max() < 1e-12 * np.abs(u).max() * n
    assert np.abs(u.mean(axis=(1, 2, 3))).max() < 1e-15
    for c in range(3):
        assert np.abs(r.dealias(u[c], 2.0) - u[c]).max() < 1e-13


def test_context_calls_reject_a_null_context():
    """Every entry point that takes a context returns MLQ_ERR_BADARG for a
    null one (no device work is attempted)."""
    lib = maxlq_b200.load_library()
    skip = {"mlq_init", "mlq_last_error", "mlq_kernel_launches", "mlq_device_bytes"}
    checked = 0
    for name, (res, args) in _capi.SIGNATURES.items():
        if name in skip or not args or args[0] is not _capi._VP or res is not ctypes.c_int:
            continue
        vals = [None]
        for a in args[1:]:
            if a in (ctypes.c_int, ctypes.c_ulonglong):
                vals.append(0)
            elif a is ctypes.c_double:
                vals.append(0.0)
            elif a is _capi.ITER_CB:
                vals.append(ctypes.cast(None, _capi.ITER_CB))  # a null callback
            else:
                vals.append(None)  # pointers: NULL
        # the text reports return the length they need, or minus a status
        want = -_capi.MLQ_ERR_BADARG if name in ("mlq_profile_report", "mlq_kernel_config") else _capi.MLQ_ERR_BADARG
        assert getattr(lib, name)(*vals) == want, name
        checked += 1
    assert checked >= 30


@pytest.mark.parametrize("order", [float("nan"), float("inf"), -3.0])
def test_noalloc_rejects_orders_that_keep_no_mode_before_any_cuda_call(order):
    # argument checks come before the first CUDA call, so they hold without a GPU
    lib = maxlq_b200.load_library()
    g = np.zeros((16, 16, 16))
    assert lib.mlq_dealias_scalar_noalloc(_capi.dptr(g), 16, order) == _capi.MLQ_ERR_BADARG


def test_fortran_module_binds_every_declared_symbol():
    # the ISO_C_BINDING module the reference's Fortran driver uses
    text = open(os.path.join(ROOT, "maxlq_b200", "fortran", "maxlq_gpu.f90")).read()
    bound = set(re.findall(r"(?:function|subroutine)\s+(mlq_\w+)\s*\(", text))
    missing = [n for n in declared_symbols() if n not in bound]
    assert not missing, missing
