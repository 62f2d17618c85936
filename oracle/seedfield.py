"""Seeded synthetic fields, written independently of the product (numpy).

TEST INFRASTRUCTURE ONLY.  Restates the project's input generator (the
reference has none; its inputs are netCDF files that are not shipped):

  u_hat(j) = A(|j|) (a + i b) / sqrt(2),  A(k) = k^-slope exp(-(k/k0)^2),
  (a, b) = Box-Muller of Philox-4x32-10(counter = (jx, jy, jz, c), key = seed),
  Hermitian on the jx = 0 plane, Leray-projected, zero mean, and only modes of
  the 2/3 dealiasing cube (|j_i| <= N/3) present.

Philox-4x32-10 follows Salmon et al., SC'11 (Random123); the known-answer
vectors of that paper's reference implementation are checked in the tests.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
    """Vectorised Philox-4x32-10.  ctr: (..., 4) uint32, key: (2,) uint32."""
    c = [np.asarray(ctr[..., i], dtype=np.uint32) for i in range(4)]
    k0, k1 = np.uint32(key[0]), np.uint32(key[1])
    with np.errstate(over="ignore"):
        for r in range(10):
            if r > 0:
                k0 = np.uint32(k0 + W0)
                k1 = np.uint32(k1 + W1)
            p0 = M0 * c[0].astype(np.uint64)
            p1 = M1 * c[2].astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & MASK).astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
    return np.stack(c, axis=-1)


def band_cut(n: int, order: float = 2.0) -> int:
    """function_ops.f90:3374-3391: largest |j| with 2 pi j <= 2 pi n/(order+1)."""
    PI = 4.0 * np.arctan2(1.0, 1.0)
    kcut = 2.0 * PI * float(n) / (order + 1.0)
    cut = -1
    for j in range(n // 2 + 1):
        if not abs(2.0 * PI * float(j)) > kcut:
            cut = j
    return cut


def seed_spectrum(n: int, seed: int, slope: float, k0: float):
    """Pruned half spectrum [3][nb kz][nb ky][nx kx], compact order 0..c, -c..-1."""
    c = band_cut(n)
    nb, nx = 2 * c + 1, c + 1
    cj = np.where(np.arange(nb) <= c, np.arange(nb), np.arange(nb) - nb)
    JZ, JY, JX = np.meshgrid(cj, cj, np.arange(nx), indexing="ij")
    neg = (JX == 0) & ((JY < 0) | ((JY == 0) & (JZ < 0)))
    GY = np.where(neg, -JY, JY)
    GZ = np.where(neg, -JZ, JZ)
    kk = np.sqrt(JX.astype(float) ** 2 + JY ** 2 + JZ ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = kk ** (-slope) * np.exp(-(kk / k0) ** 2) / np.sqrt(2.0)
    amp[0, 0, 0] = 0.0
    key = np.array([seed & 0xFFFFFFFF, seed >> 32], dtype=np.uint64).astype(np.uint32)
    out = np.zeros((3, nb, nb, nx), dtype=np.complex128)
    for comp in range(3):
        ctr = np.stack([JX.astype(np.int64) & 0xFFFFFFFF, GY.astype(np.int64) & 0xFFFFFFFF,
                        GZ.astype(np.int64) & 0xFFFFFFFF, np.full(JX.shape, comp)], axis=-1).astype(np.uint32)
        r = philox4x32_10(ctr, key).astype(np.uint64)
        m1 = ((r[..., 0] << np.uint64(32)) | r[..., 1]) >> np.uint64(11)
        m2 = ((r[..., 2] << np.uint64(32)) | r[..., 3]) >> np.uint64(11)
        u1 = (m1.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
        u2 = (m2.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
        rr = np.sqrt(-2.0 * np.log(u1))
        th = 2.0 * np.pi * u2
        a, b = rr * np.cos(th), rr * np.sin(th)
        b = np.where(neg, -b, b)
        out[comp] = amp * (a + 1j * b)
    # Leray projection with the integer wavevector
    jv = [JX.astype(float), JY.astype(float), JZ.astype(float)]
    with np.errstate(divide="ignore", invalid="ignore"):
        div = (jv[0] * out[0] + jv[1] * out[1] + jv[2] * out[2]) / kk ** 2
    div[0, 0, 0] = 0.0
    for comp in range(3):
        out[comp] = out[comp] - jv[comp] * div
    out[:, 0, 0, 0] = 0.0
    return out, c


def spectrum_to_field(spec: np.ndarray, n: int) -> np.ndarray:
    """Physical field u(x) = sum_j u_hat(j) e^{2 pi i j.x} from a pruned half spectrum."""
    nb, nx = spec.shape[-3], spec.shape[-1]
    c = nx - 1
    fi = np.where(np.arange(nb) <= c, np.arange(nb), n - nb + np.arange(nb))
    full = np.zeros(spec.shape[:-3] + (n, n, n // 2 + 1), dtype=np.complex128)
    full[..., fi[:, None, None], fi[None, :, None], np.arange(nx)[None, None, :]] = spec
    return np.fft.irfftn(full, s=(n, n, n), axes=(-3, -2, -1)) * float(n) ** 3


def seed_field(n: int, seed: int = 0, slope: float = 2.0, k0: float = 4.0) -> np.ndarray:
    spec, _ = seed_spectrum(n, seed, slope, k0)
    return spectrum_to_field(spec, n)
