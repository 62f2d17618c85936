"""Independent numpy transcription of the reference's hot-path operators.

TEST INFRASTRUCTURE ONLY.  A second, separately written restatement of the
Fortran (numpy/pocketfft FFTs instead of the C++ oracle's own FFT), used to
cross-check oracle/mlq_oracle.cpp at small N and to generate the committed
golden fixtures under tests/golden/.  Same conventions as oracle.py: fields
are float64 arrays [c, z, y, x]; reference-order semantics (each operator is
a c2c FFT round trip followed by REAL()).

Parity unpinned (the reference's own outputs are unavailable); agreement with
the C++ oracle is what the two transcriptions establish.

Citations are to the reference project's function_ops.f90 (FO) and
optimization.f90 (OPT).
"""
from __future__ import annotations

import numpy as np

MACH_EPSILON = 2.0e-16


class RefNumpy:
    def __init__(self, n, q, B=1.0, visc=1.0, lambda1=0.1, use_e_u=None, dealias_e_u=True, to_dealias=True,
                 workers=None):
        self.n, self.q, self.B = n, float(q), float(B)
        self.workers = workers  # scipy.fft threads (None: numpy.fft, single thread)
        self.visc, self.lambda1 = visc, lambda1
        self.use_e_u = (q < 4.0 - MACH_EPSILON) if use_e_u is None else use_e_u
        self.dealias_e_u, self.to_dealias = dealias_e_u, to_dealias
        self.PI = 4.0 * np.arctan2(1.0, 1.0)
        i = np.arange(n)
        k = np.where(i <= n // 2, 2.0 * self.PI * i, 2.0 * self.PI * (i - n))
        self.k1 = k
        # broadcastable wavenumbers for [z, y, x] arrays
        self.KX = k[None, None, :]
        self.KY = k[None, :, None]
        self.KZ = k[:, None, None]
        self.KSQ = self.KX ** 2 + self.KY ** 2 + self.KZ ** 2
        self.dV = 1.0 / float(n) ** 3

    # fftfwd / fftbwd (fftwfunction.f90:62-113)
    def fwd(self, f):
        if self.workers:
            import scipy.fft
            return scipy.fft.fftn(f.astype(np.complex128), workers=self.workers, overwrite_x=True)
        return np.fft.fftn(f.astype(np.complex128))

    def bwd(self, fh):
        if self.workers:
            import scipy.fft
            return scipy.fft.ifftn(fh, workers=self.workers)
        return np.fft.ifftn(fh)  # ifftn already divides by N^3

    def dealias(self, g, order):  # FO 3332-3398
        if not self.to_dealias:
            return g
        kcut = 2.0 * self.PI * float(self.n) / (order + 1.0)
        keep = np.abs(self.k1) <= kcut
        m = keep[:, None, None] & keep[None, :, None] & keep[None, None, :]
        return self.bwd(self.fwd(g) * m).real

    def gradient(self, f):  # FO 3147-3195
        fh = self.fwd(f)
        return np.stack([self.bwd(1j * K * fh).real for K in (self.KX, self.KY, self.KZ)])

    def divergence(self, u):  # FO 3200-3243
        h = 1j * self.KX * self.fwd(u[0]) + 1j * self.KY * self.fwd(u[1]) + 1j * self.KZ * self.fwd(u[2])
        return self.bwd(h).real

    def laplacian(self, u):  # FO 3248-3282
        return np.stack([self.bwd(-self.KSQ * self.fwd(c)).real for c in u])

    def solve_poisson(self, f, l=1.0):  # FO 1951-1996
        fh = self.fwd(f)
        with np.errstate(divide="ignore", invalid="ignore"):
            ph = np.where(self.KSQ == 0, 0.0, -fh / (l ** 2 * self.KSQ))
        return self.bwd(ph).real

    def gk(self, g, k):  # FO 2281-2319
        if k + MACH_EPSILON < 0:
            with np.errstate(divide="ignore", invalid="ignore"):
                return np.where(np.abs(g) < MACH_EPSILON, 0.0, g ** k)
        if k + MACH_EPSILON < 2.0:
            return self.dealias(g ** k, k)
        g2 = self.dealias(g * g, 2.0)
        return self.dealias(g2 * self.gk(g, k - 2.0), 2.0)

    def calc_uk(self, u, k):  # FO 2324-2343
        s = self.dealias((u ** 2).sum(0), 2.0)
        s = np.where(s <= 0.0, 0.0, np.sqrt(np.maximum(s, 0.0)))
        return self.gk(s, k)

    def unit_vector(self, u):  # FO 1775-1791, 1822-1858
        nrm = np.sqrt(np.abs(self.dealias((u ** 2).sum(0), 2.0)))
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(nrm[None] < MACH_EPSILON, 0.0, u / nrm[None])

    def grad_tensor(self, u):  # G[i, j] = d_j u_i
        return np.stack([self.gradient(c) for c in u])

    def _dealias_e(self):
        return self.to_dealias and ((not self.use_e_u) or self.dealias_e_u)

    def vgraduvgradu(self, u, v):  # FO 2165-2218
        G = self.grad_tensor(u)
        vg = np.einsum("i...,ij...->j...", v, G)
        if self._dealias_e():
            vg = np.stack([self.dealias(c, 2.0) for c in vg])
        return self.dealias((vg ** 2).sum(0), 2.0)

    def vvgradu(self, u, v):  # FO 2001-2064
        G = self.grad_tensor(u)
        aux = np.einsum("i...,ij...->j...", v, G)
        if self._dealias_e():
            aux = np.stack([self.dealias(c, 2.0) for c in aux])
        res = (v * aux).sum(0)
        return self.dealias(res, 2.0) if self._dealias_e() else res

    def nabla_u_nabla_ut(self, u):  # FO 1912-1945
        G = self.grad_tensor(u)
        return self.dealias(np.einsum("ij...,ji...->...", G, G), 2.0)

    def nabla_mod_squared(self, u):  # FO 2366-2389
        G = self.grad_tensor(u)
        return self.dealias((G ** 2).sum((0, 1)), 2.0)

    def l2(self, f, g):  # FO 3427-3437
        return float((f * g).sum() * self.dV)

    def hl(self, f, g):  # FO 3462-3483
        order = 1.5 - 1.0 / self.q
        w = 1.0 + (self.lambda1 * np.sqrt(self.KSQ)) ** order
        return self.l2(self.bwd(w * self.fwd(f)).real, self.bwd(w * self.fwd(g)).real)

    def field_inner(self, f, g, htype="L2"):  # FO 3557-3577
        ip = self.l2 if htype == "L2" else self.hl
        return sum(ip(f[i], g[i]) for i in range(3))

    def R_parts(self, u):  # FO 1304-1358
        q, nu = self.q, self.visc
        a2 = self.calc_uk(u, q - 2.0)
        R1 = -nu * self.l2(a2, self.nabla_mod_squared(u))
        e = self.unit_vector(u)
        if self.use_e_u:
            R2 = -(q - 2.0) * nu * self.l2(a2, self.vgraduvgradu(u, e))
            mult, v = a2, e
        else:
            a4 = self.calc_uk(u, q - 4.0)
            R2 = -(q - 2.0) * nu * self.l2(a4, self.vgraduvgradu(u, u))
            mult, v = a4, u
        p = self.solve_poisson(-self.nabla_u_nabla_ut(u), 1.0)
        aux = self.dealias(p * mult, 2.0)
        R3 = (q - 2.0) * self.l2(aux, self.vvgradu(u, v))
        return np.array([R1 + R2 + R3, R1 + R2, R3])

    def lq_norm(self, u):  # FO 1675-1692
        a = self.calc_uk(u, self.q / 2.0)
        return self.l2(a, a) ** (1.0 / self.q)

    def rescale(self, u, B=None):  # FO 1699-1709
        return (self.B if B is None else B) / self.lq_norm(u) * u

    def divavg_free(self, f):  # FO 2843-2918
        dh = self.fwd(self.divergence(f))
        uh = np.stack([self.fwd(c) for c in f])
        nz = self.KSQ > MACH_EPSILON
        with np.errstate(divide="ignore", invalid="ignore"):
            gp = np.stack([np.where(nz, -(1j * K) * dh / self.KSQ, 0.0) for K in (self.KX, self.KY, self.KZ)])
        uh = np.where(nz[None], uh, 0.0)
        return np.stack([self.bwd(uh[i]).real - self.bwd(gp[i]).real for i in range(3)])

    def hilbert(self, g, order):  # FO 3583-3627
        w = 1.0 / (1.0 + (self.lambda1 * np.sqrt(self.KSQ)) ** (2.0 * order))
        return np.stack([self.bwd(w * self.fwd(c)).real for c in g])

    def normal_l2(self, u):  # FO 984-1006
        nrm = self.lq_norm(u)
        a = self.calc_uk(u, self.q - 2.0)
        out = np.stack([a * c for c in u])
        if self.to_dealias and self.q - 2.0 > MACH_EPSILON:
            out = np.stack([self.dealias(c, 2.0) for c in out])
        return nrm ** (1.0 - self.q) * out

    def vector_transport(self, u, eta, xi, q=None, B=None):  # FO 1716-1768
        q = self.q if q is None else q
        B = self.B if B is None else B
        w = u + eta
        a = self.calc_uk(w, q - 2.0)
        aux = np.stack([a * c for c in w])
        if self.to_dealias and q - 2.0 > MACH_EPSILON:
            aux = np.stack([self.dealias(c, 2.0) for c in aux])
        ir = self.field_inner(aux, xi)
        ln = self.lq_norm(w)
        return B / ln * (xi - ln ** (-q) * ir * w)

    def grad_l2(self, u):  # FO 1066-1211
        q, nu = self.q, self.visc
        a2 = self.calc_uk(u, q - 2.0)
        p = self.solve_poisson(-self.nabla_u_nabla_ut(u), 1.0)
        gp = self.gradient(p)
        du = self.laplacian(u)
        if self.use_e_u:
            e = self.unit_vector(u)
            aux2 = (e * (nu * du - gp)).sum(0)
            if self.to_dealias and self.dealias_e_u:
                aux2 = self.dealias(aux2, 2.0)
            aux2 = self.dealias(a2 * aux2, 2.0)
            a3 = aux2[None] * e
            if self.to_dealias and self.dealias_e_u:
                a3 = np.stack([self.dealias(c, 2.0) for c in a3])
        else:
            aux2 = self.dealias((u * (nu * du - gp)).sum(0), 2.0)
            aux2 = self.dealias(self.calc_uk(u, q - 4.0) * aux2, 2.0)
            a3 = np.stack([self.dealias(aux2 * c, 2.0) for c in u])
        uq2u = np.stack([self.dealias(a2 * c, 2.0) for c in u])
        a4 = self.solve_poisson(self.divergence(uq2u), 1.0)
        a4v = self.gradient(a4)
        G = self.grad_tensor(u)  # G[k, i] = d_i u_k
        a5 = np.stack([self.dealias((G[:, i] * a4v).sum(0), 2.0) for i in range(3)])
        a7 = self.laplacian(uq2u)
        a4b = np.stack([self.dealias(a2 * c, 2.0) for c in gp])
        a6 = np.stack([self.dealias(a2 * c, 2.0) for c in du])
        return (q - 2.0) * a3 - a4b + 2.0 * a5 + nu * a6 + nu * a7

    def eval_J(self, u, mode="maxdLqdt"):  # OPT 520-547
        if mode == "maxdLqdt":
            return self.R_parts(u)[0]
        if mode == "LineMin":
            return -1.0 * self.R_parts(self.rescale(u))[0]
        return self.lq_norm(u)
