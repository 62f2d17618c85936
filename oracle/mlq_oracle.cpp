// mlq_oracle.cpp -- CPU FP64 restatement of maxLq's CG hot path, reference order.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product (see mlq_oracle.h).
// Each function cites the Fortran routine it restates (paths are relative to
// the reference project root).  Arithmetic follows the Fortran expression
// order where it matters for masks and thresholds.
#include "mlq_oracle.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

const double MACH_EPSILON = 2.0e-16;  // global_variables.f90:28
const double TAU_MAX = 1.0e2;         // global_variables.f90:29

// ---------------------------------------------------------------------------
// 1D mixed-radix Stockham FFT (radices 4, 2, 3, 5, generic), applied to B
// interleaved lines at once (element p of line b at x[p*B + b]) so that the
// strided y and z lines of a 3D array are transformed in cache-friendly tiles
// of B neighbouring columns.  The oracle's own FFT: FFTW is not vendored by
// the reference (makefile:20-21), so parity at this boundary is the
// mathematical DFT (checked against numpy's pocketfft in the tests).
// Complex products are written out in real arithmetic.
// ---------------------------------------------------------------------------
struct Fft1D {
    int n = 0;
    std::vector<int> radix, ns;          // radix and span of every stage
    std::vector<std::vector<cplx>> stw;  // stage twiddles [k*(R-1) + r-1] = exp(-2 pi i r k / (ns R))
    std::vector<std::vector<cplx>> roots;  // roots[R][m] = exp(-2 pi i m / R) for the generic radices

    static cplx expi(long num, long den) {  // exp(-2 pi i num / den), angle reduced in integers
        long k = ((num % den) + den) % den;
        const double a = 2.0 * M_PI * (double)k / (double)den;
        return cplx(std::cos(a), -std::sin(a));
    }
    void init(int nn) {
        n = nn;
        radix.clear();
        int m = n;
        while (m % 4 == 0) { radix.push_back(4); m /= 4; }
        while (m % 2 == 0) { radix.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2) {
            while (m % p == 0) { radix.push_back(p); m /= p; }
        }
        ns.clear();
        stw.clear();
        roots.assign(64, {});
        int span = 1;
        for (int R : radix) {
            ns.push_back(span);
            std::vector<cplx> t((size_t)span * (R - 1));
            for (int k = 0; k < span; ++k)
                for (int r = 1; r < R; ++r) t[(size_t)k * (R - 1) + r - 1] = expi((long)r * k, (long)span * R);
            stw.push_back(t);
            if (R != 2 && R != 4 && R < 64 && roots[R].empty()) {
                roots[R].resize(R);
                for (int q = 0; q < R; ++q) roots[R][q] = expi(q, R);
            }
            span *= R;
        }
    }
    // sign -1: forward exp(-i...), +1: backward exp(+i...).  Unnormalised.
    // work holds n*B elements.
    void exec_batch(cplx* x, cplx* work, int B, int sign) const {
        double* src = reinterpret_cast<double*>(x);
        double* dst = reinterpret_cast<double*>(work);
        const double sg = (double)sign;  // conj of the forward twiddles when +1
        for (size_t s = 0; s < radix.size(); ++s) {
            const int R = radix[s], NS = ns[s], nr = n / R;
            const double* tw = reinterpret_cast<const double*>(stw[s].data());
            for (int j = 0; j < nr; ++j) {
                const int k = j % NS;
                const long od = ((long)(j / NS) * NS * R + k) * B;
                const double* twk = tw + 2 * (long)k * (R - 1);
                if (R == 4) {
                    double wr[3], wi[3];
                    for (int r = 0; r < 3; ++r) {
                        wr[r] = twk[2 * r];
                        wi[r] = sign < 0 ? twk[2 * r + 1] : -twk[2 * r + 1];
                    }
                    for (int b = 0; b < B; ++b) {
                        double vr[4], vi[4];
                        for (int r = 0; r < 4; ++r) {
                            const long is = 2 * ((long)(j + r * nr) * B + b);
                            vr[r] = src[is];
                            vi[r] = src[is + 1];
                        }
                        if (NS > 1) {
                            for (int r = 1; r < 4; ++r) {
                                const double ar = vr[r], ai = vi[r];
                                vr[r] = ar * wr[r - 1] - ai * wi[r - 1];
                                vi[r] = ar * wi[r - 1] + ai * wr[r - 1];
                            }
                        }
                        const double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
                        const double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
                        const double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
                        const double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
                        // o1 = d0 + sign * i * d1, o3 = d0 - sign * i * d1
                        const long o = 2 * (od + b);
                        const long st = 2 * (long)NS * B;
                        dst[o] = s0r + s1r;
                        dst[o + 1] = s0i + s1i;
                        dst[o + st] = d0r - sg * d1i;
                        dst[o + st + 1] = d0i + sg * d1r;
                        dst[o + 2 * st] = s0r - s1r;
                        dst[o + 2 * st + 1] = s0i - s1i;
                        dst[o + 3 * st] = d0r + sg * d1i;
                        dst[o + 3 * st + 1] = d0i - sg * d1r;
                    }
                } else if (R == 2) {
                    const double wr = twk[0], wi = sign < 0 ? twk[1] : -twk[1];
                    for (int b = 0; b < B; ++b) {
                        const long i0 = 2 * ((long)j * B + b), i1 = 2 * ((long)(j + nr) * B + b);
                        double ar = src[i1], ai = src[i1 + 1];
                        if (NS > 1) {
                            const double tr = ar * wr - ai * wi;
                            ai = ar * wi + ai * wr;
                            ar = tr;
                        }
                        const long o = 2 * (od + b), st = 2 * (long)NS * B;
                        dst[o] = src[i0] + ar;
                        dst[o + 1] = src[i0 + 1] + ai;
                        dst[o + st] = src[i0] - ar;
                        dst[o + st + 1] = src[i0 + 1] - ai;
                    }
                } else {
                    const std::vector<cplx>& rt = roots[R];
                    cplx v[64];
                    for (int b = 0; b < B; ++b) {
                        for (int r = 0; r < R; ++r) {
                            const long is = 2 * ((long)(j + r * nr) * B + b);
                            double ar = src[is], ai = src[is + 1];
                            if (r > 0 && NS > 1) {
                                const double wr = twk[2 * (r - 1)];
                                const double wi = sign < 0 ? twk[2 * (r - 1) + 1] : -twk[2 * (r - 1) + 1];
                                const double tr = ar * wr - ai * wi;
                                ai = ar * wi + ai * wr;
                                ar = tr;
                            }
                            v[r] = cplx(ar, ai);
                        }
                        for (int m = 0; m < R; ++m) {
                            double accr = 0.0, acci = 0.0;
                            for (int r = 0; r < R; ++r) {
                                const cplx w = rt[(long)r * m % R];
                                const double wr = w.real(), wi = sign < 0 ? w.imag() : -w.imag();
                                accr += v[r].real() * wr - v[r].imag() * wi;
                                acci += v[r].real() * wi + v[r].imag() * wr;
                            }
                            const long o = 2 * (od + (long)m * NS * B + b);
                            dst[o] = accr;
                            dst[o + 1] = acci;
                        }
                    }
                }
            }
            std::swap(src, dst);
        }
        double* xd = reinterpret_cast<double*>(x);
        if (src != xd) std::memcpy(xd, src, sizeof(double) * 2 * (size_t)n * B);
    }
};

}  // namespace

struct orc_ctx {
    orc_params p;
    int n;
    long n3;
    double dV, PI;
    std::vector<double> K;  // K1 = K2 = K3 (initialize.f90:170-192)
    Fft1D fft;
    int n_evals = 0;
};

namespace {

inline long IDX(const orc_ctx* c, int x, int y, int z) {
    return ((long)z * c->n + y) * c->n + x;
}

// 3D c2c over [z][y][x], all three axes; sign as Fft1D.  y and z lines are
// transformed in tiles of TB neighbouring x columns.
void fft3(orc_ctx* c, cplx* a, int sign) {
    const int n = c->n;
    int TB = 16;
    while (n % TB) TB /= 2;
    const int ntile = n / TB;
#pragma omp parallel
    {
        std::vector<cplx> buf((size_t)n * TB), work((size_t)n * TB);
        // x lines (contiguous)
#pragma omp for collapse(2) schedule(static)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y) c->fft.exec_batch(a + IDX(c, 0, y, z), work.data(), 1, sign);
        // y lines, TB columns at a time
#pragma omp for collapse(2) schedule(static)
        for (int z = 0; z < n; ++z)
            for (int t = 0; t < ntile; ++t) {
                const int x0 = t * TB;
                for (int y = 0; y < n; ++y)
                    std::memcpy(&buf[(size_t)y * TB], a + IDX(c, x0, y, z), sizeof(cplx) * TB);
                c->fft.exec_batch(buf.data(), work.data(), TB, sign);
                for (int y = 0; y < n; ++y)
                    std::memcpy(a + IDX(c, x0, y, z), &buf[(size_t)y * TB], sizeof(cplx) * TB);
            }
        // z lines
#pragma omp for collapse(2) schedule(static)
        for (int y = 0; y < n; ++y)
            for (int t = 0; t < ntile; ++t) {
                const int x0 = t * TB;
                for (int z = 0; z < n; ++z)
                    std::memcpy(&buf[(size_t)z * TB], a + IDX(c, x0, y, z), sizeof(cplx) * TB);
                c->fft.exec_batch(buf.data(), work.data(), TB, sign);
                for (int z = 0; z < n; ++z)
                    std::memcpy(a + IDX(c, x0, y, z), &buf[(size_t)z * TB], sizeof(cplx) * TB);
            }
    }
}

// fftfwd (fftwfunction.f90:62-93): unnormalised forward.  The NaN scan with
// `stop 1` (78-89) is mirrored by the caller-visible status of the product,
// not here.
void fftfwd(orc_ctx* c, cplx* a) { fft3(c, a, -1); }

// fftbwd (fftwfunction.f90:98-113): backward then /product(n).
void fftbwd(orc_ctx* c, cplx* a) {
    fft3(c, a, +1);
    const double s = (double)c->n * (double)c->n * (double)c->n;
#pragma omp parallel for
    for (long i = 0; i < c->n3; ++i) a[i] /= s;
}

typedef std::vector<double> RV;
typedef std::vector<cplx> CV;

CV to_complex(const orc_ctx* c, const double* f) {
    CV a(c->n3);
#pragma omp parallel for
    for (long i = 0; i < c->n3; ++i) a[i] = cplx(f[i], 0.0);
    return a;
}
void real_part(const orc_ctx* c, const CV& a, double* f) {
#pragma omp parallel for
    for (long i = 0; i < c->n3; ++i) f[i] = a[i].real();
}

inline double Kx(const orc_ctx* c, int i) { return c->K[i]; }

// dealiasing_cutoff_scalar_complex (function_ops.f90:3358-3398): zero modes
// with max(|K1|,|K2|,|K3|) > 2 pi n / (order+1).
void dealias_cut(orc_ctx* c, CV& f, double order) {
    const double kcut = 2.0 * c->PI * (double)c->n / (order + 1.0);
    const int n = c->n;
    std::vector<char> keep(n);
    for (int i = 0; i < n; ++i) keep[i] = std::fabs(c->K[i]) > kcut ? 0 : 1;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x)
                if (!(keep[x] && keep[y] && keep[z])) f[IDX(c, x, y, z)] = 0.0;
}

// dealias_scalar (function_ops.f90:3332-3350)
void dealias_scalar(orc_ctx* c, double* g, double order) {
    CV a = to_complex(c, g);
    fftfwd(c, a.data());
    dealias_cut(c, a, order);
    fftbwd(c, a.data());
    real_part(c, a, g);
}

inline void maybe_dealias(orc_ctx* c, double* g, double order) {
    if (c->p.to_dealias) dealias_scalar(c, g, order);
}

// gradient (function_ops.f90:3147-3195): grad is [3][n3]
void gradient(orc_ctx* c, const double* u, double* grad) {
    const int n = c->n;
    CV fu = to_complex(c, u);
    fftfwd(c, fu.data());
    for (int d = 0; d < 3; ++d) {
        CV g(c->n3);
#pragma omp parallel for collapse(2)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    double k = d == 0 ? Kx(c, x) : (d == 1 ? Kx(c, y) : Kx(c, z));
                    g[IDX(c, x, y, z)] = cplx(0.0, k) * fu[IDX(c, x, y, z)];
                }
        fftbwd(c, g.data());
        real_part(c, g, grad + d * c->n3);
    }
}

// divergence (function_ops.f90:3200-3243)
void divergence(orc_ctx* c, const double* u, double* div) {
    const int n = c->n;
    CV uh[3];
    for (int d = 0; d < 3; ++d) {
        uh[d] = to_complex(c, u + d * c->n3);
        fftfwd(c, uh[d].data());
    }
    CV dh(c->n3);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                long i = IDX(c, x, y, z);
                dh[i] = cplx(0.0, Kx(c, x)) * uh[0][i] + cplx(0.0, Kx(c, y)) * uh[1][i] +
                        cplx(0.0, Kx(c, z)) * uh[2][i];
            }
    fftbwd(c, dh.data());
    real_part(c, dh, div);
}

inline double ksq_of(const orc_ctx* c, int x, int y, int z) {
    return Kx(c, x) * Kx(c, x) + Kx(c, y) * Kx(c, y) + Kx(c, z) * Kx(c, z);
}

// laplacian (function_ops.f90:3248-3282), in place on a vector field
void laplacian(orc_ctx* c, double* f) {
    const int n = c->n;
    for (int d = 0; d < 3; ++d) {
        CV a = to_complex(c, f + d * c->n3);
        fftfwd(c, a.data());
#pragma omp parallel for collapse(2)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) a[IDX(c, x, y, z)] *= -ksq_of(c, x, y, z);
        fftbwd(c, a.data());
        real_part(c, a, f + d * c->n3);
    }
}

// solve_poisson (function_ops.f90:1951-1996): l^2 Delta phi = f, k=0 -> 0
void solve_poisson(orc_ctx* c, const double* f, double l, double* phi) {
    const int n = c->n;
    CV a = to_complex(c, f);
    fftfwd(c, a.data());
    const double l2 = std::pow(l, 2.0);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                long i = IDX(c, x, y, z);
                double ksq = ksq_of(c, x, y, z);
                a[i] = ksq == 0.0 ? cplx(0.0, 0.0) : -a[i] / (l2 * ksq);
            }
    fftbwd(c, a.data());
    real_part(c, a, phi);
}

// calc_gk_order2 (function_ops.f90:2281-2319), recursive
void calc_gk_order2(orc_ctx* c, const double* g, double k, double* gk) {
    const long n3 = c->n3;
    if (k + MACH_EPSILON < 0.0) {
#pragma omp parallel for
        for (long i = 0; i < n3; ++i) gk[i] = std::fabs(g[i]) < MACH_EPSILON ? 0.0 : std::pow(g[i], k);
    } else if (k + MACH_EPSILON < 2.0) {
#pragma omp parallel for
        for (long i = 0; i < n3; ++i) gk[i] = std::pow(g[i], k);
        maybe_dealias(c, gk, k);
    } else {
        RV g2(n3), gkm2(n3);
#pragma omp parallel for
        for (long i = 0; i < n3; ++i) g2[i] = g[i] * g[i];
        maybe_dealias(c, g2.data(), 2.0);
        calc_gk_order2(c, g, k - 2.0, gkm2.data());
#pragma omp parallel for
        for (long i = 0; i < n3; ++i) gk[i] = g2[i] * gkm2[i];
        maybe_dealias(c, gk, 2.0);
    }
}

// calc_uk (function_ops.f90:2324-2343)
void calc_uk(orc_ctx* c, const double* u, double k, double* uk) {
    const long n3 = c->n3;
    RV s(n3);
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) {
        double a = u[i], b = u[n3 + i], d = u[2 * n3 + i];
        s[i] = a * a + b * b + d * d;
    }
    maybe_dealias(c, s.data(), 2.0);
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) s[i] = s[i] <= 0.0 ? 0.0 : std::pow(s[i], 0.5);
    calc_gk_order2(c, s.data(), k, uk);
}

// calc_pointwiseVectorNorm (1775-1791) + calc_unitVectorInUdirection (1822-1858)
void unit_vector(orc_ctx* c, const double* u, double* e) {
    const long n3 = c->n3;
    RV nrm(n3);
#pragma omp parallel for
    for (long i = 0; i < n3; ++i)
        nrm[i] = u[i] * u[i] + u[n3 + i] * u[n3 + i] + u[2 * n3 + i] * u[2 * n3 + i];
    maybe_dealias(c, nrm.data(), 2.0);
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) nrm[i] = std::sqrt(std::fabs(nrm[i]));
    for (int d = 0; d < 3; ++d)
#pragma omp parallel for
        for (long i = 0; i < n3; ++i) e[d * n3 + i] = nrm[i] < MACH_EPSILON ? 0.0 : u[d * n3 + i] / nrm[i];
}

// gradU[i][j] = partial_j u_i as 9 scalar fields
RV grad_tensor(orc_ctx* c, const double* u) {
    RV g(9 * c->n3);
    for (int i = 0; i < 3; ++i) gradient(c, u + i * c->n3, g.data() + 3 * i * c->n3);
    return g;
}
inline const double* GU(const RV& g, const orc_ctx* c, int i, int j) { return g.data() + (3 * i + j) * c->n3; }

// calc_nablaUnablaUt (1912-1945): sum_ij d_j u_i d_i u_j
void nabla_u_nabla_ut(orc_ctx* c, const double* u, double* out) {
    RV g = grad_tensor(c, u);
    const long n3 = c->n3;
#pragma omp parallel for
    for (long p = 0; p < n3; ++p) {
        double s = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) s += GU(g, c, j, i)[p] * GU(g, c, i, j)[p];
        out[p] = s;
    }
    maybe_dealias(c, out, 2.0);
}

bool dealias_for_e_u(const orc_ctx* c) {
    if (!c->p.to_dealias) return false;
    return !c->p.use_e_u || c->p.dealias_e_u;
}

// calc_vvgradu (2001-2064): v . (v . nabla) u
void vvgradu(orc_ctx* c, const double* u, const double* v, double* res) {
    RV g = grad_tensor(c, u);
    const long n3 = c->n3;
    RV aux(3 * n3);
#pragma omp parallel for
    for (long p = 0; p < n3; ++p)
        for (int jj = 0; jj < 3; ++jj) {
            double s = 0.0;
            for (int ii = 0; ii < 3; ++ii) s += v[ii * n3 + p] * GU(g, c, ii, jj)[p];
            aux[jj * n3 + p] = s;
        }
    if (dealias_for_e_u(c))
        for (int d = 0; d < 3; ++d) dealias_scalar(c, aux.data() + d * n3, 2.0);
#pragma omp parallel for
    for (long p = 0; p < n3; ++p) {
        double s = 0.0;
        for (int jj = 0; jj < 3; ++jj) s += v[jj * n3 + p] * aux[jj * n3 + p];
        res[p] = s;
    }
    if (dealias_for_e_u(c)) dealias_scalar(c, res, 2.0);
}

// calc_vgraduvgradu (2165-2218): v_i d_j u_i v_k d_j u_k
void vgraduvgradu(orc_ctx* c, const double* u, const double* v, double* res) {
    RV g = grad_tensor(c, u);
    const long n3 = c->n3;
    RV vg(3 * n3);
#pragma omp parallel for
    for (long p = 0; p < n3; ++p)
        for (int jj = 0; jj < 3; ++jj) {
            double s = 0.0;
            for (int ii = 0; ii < 3; ++ii) s += v[ii * n3 + p] * GU(g, c, ii, jj)[p];
            vg[jj * n3 + p] = s;
        }
    if (dealias_for_e_u(c))
        for (int d = 0; d < 3; ++d) dealias_scalar(c, vg.data() + d * n3, 2.0);
#pragma omp parallel for
    for (long p = 0; p < n3; ++p) {
        double s = 0.0;
        for (int jj = 0; jj < 3; ++jj) s += vg[jj * n3 + p] * vg[jj * n3 + p];
        res[p] = s;
    }
    maybe_dealias(c, res, 2.0);
}

// calc_nablaModSquared (2366-2389)
void nabla_mod_squared(orc_ctx* c, const double* u, double* out) {
    const long n3 = c->n3;
    std::memset(out, 0, sizeof(double) * n3);
    RV g(3 * n3);
    for (int i = 0; i < 3; ++i) {
        gradient(c, u + i * n3, g.data());
#pragma omp parallel for
        for (long p = 0; p < n3; ++p)
            for (int j = 0; j < 3; ++j) out[p] += g[j * n3 + p] * g[j * n3 + p];
    }
    maybe_dealias(c, out, 2.0);
}

// inner_product "L2" (3427-3437)
double inner_l2(const orc_ctx* c, const double* f, const double* g) {
    double s = 0.0;
    // fixed (serial) order: the reference sums i1 fastest, one rank
    for (long i = 0; i < c->n3; ++i) s += f[i] * g[i];
    return s * c->dV;
}

// inner_product "H_l^(3/2-1/q)" (3462-3483)
double inner_hl(orc_ctx* c, const double* f, const double* g) {
    const int n = c->n;
    CV fh = to_complex(c, f), gh = to_complex(c, g);
    fftfwd(c, fh.data());
    fftfwd(c, gh.data());
    const double order = (3.0 / 2.0) - (1.0 / c->p.q);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                long i = IDX(c, x, y, z);
                double ks = std::sqrt(ksq_of(c, x, y, z));
                double factor = 1.0 + std::pow(c->p.lambda1 * ks, order);
                fh[i] *= factor;
                gh[i] *= factor;
            }
    fftbwd(c, fh.data());
    fftbwd(c, gh.data());
    RV fa(c->n3), ga(c->n3);
    real_part(c, fh, fa.data());
    real_part(c, gh, ga.data());
    return inner_l2(c, fa.data(), ga.data());
}

double inner(orc_ctx* c, const double* f, const double* g, int htype) {
    return htype ? inner_hl(c, f, g) : inner_l2(c, f, g);
}

// global_summed_field_inner_product (3557-3577)
double field_inner(orc_ctx* c, const double* f, const double* g, int htype) {
    double s = 0.0;
    for (int d = 0; d < 3; ++d) s += inner(c, f + d * c->n3, g + d * c->n3, htype);
    return s;
}

// calc_local_dLqdt_inclParts (1304-1358); one rank so local == global (1392-1405)
void R_parts(orc_ctx* c, const double* u, double out[3]) {
    const long n3 = c->n3;
    const double q = c->p.q, nu = c->p.visc, vc = c->p.visc_coef, pc = c->p.press_coef;
    RV a_q2(n3), aux(n3), e(3 * n3), a_q4(n3), p(n3), tmp(n3);
    calc_uk(c, u, q - 2.0, a_q2.data());
    nabla_mod_squared(c, u, aux.data());
    double R1 = -vc * nu * inner_l2(c, a_q2.data(), aux.data());
    unit_vector(c, u, e.data());  // computed unconditionally (1323)
    double R2;
    if (c->p.use_e_u) {
        vgraduvgradu(c, u, e.data(), aux.data());
        R2 = -vc * (q - 2.0) * nu * inner_l2(c, a_q2.data(), aux.data());
    } else {
        calc_uk(c, u, q - 4.0, a_q4.data());
        vgraduvgradu(c, u, u, aux.data());
        R2 = -vc * (q - 2.0) * nu * inner_l2(c, a_q4.data(), aux.data());
    }
    nabla_u_nabla_ut(c, u, aux.data());
    #pragma omp parallel for
    for (long i = 0; i < n3; ++i) tmp[i] = -aux[i];
    solve_poisson(c, tmp.data(), 1.0, p.data());
    double R3;
    const double* mult = c->p.use_e_u ? a_q2.data() : a_q4.data();
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) aux[i] = p[i] * mult[i];
    maybe_dealias(c, aux.data(), 2.0);
    vvgradu(c, u, c->p.use_e_u ? e.data() : u, tmp.data());
    R3 = pc * (q - 2.0) * inner_l2(c, aux.data(), tmp.data());
    out[0] = R1 + R2 + R3;
    out[1] = R1 + R2;
    out[2] = R3;
}

// calc_global_Lq_norm (1675-1692)
double lq_norm(orc_ctx* c, const double* u) {
    RV a(c->n3);
    calc_uk(c, u, c->p.q / 2.0, a.data());
    double ip = inner_l2(c, a.data(), a.data());
    return std::pow(ip, 1.0 / c->p.q);
}

// rescaleLqNorm (1699-1709)
void rescale(orc_ctx* c, double* u, double B) {
    double nrm = lq_norm(c, u);
    const long m = 3 * c->n3;
    #pragma omp parallel for
    for (long i = 0; i < m; ++i) u[i] = B / nrm * u[i];
}

// divAvg_free (2843-2918)
void divavg_free(orc_ctx* c, double* f) {
    const int n = c->n;
    const long n3 = c->n3;
    RV div(n3);
    divergence(c, f, div.data());
    CV dh = to_complex(c, div.data());
    fftfwd(c, dh.data());
    CV uh[3], gp[3];
    for (int d = 0; d < 3; ++d) {
        uh[d] = to_complex(c, f + d * n3);
        fftfwd(c, uh[d].data());
        gp[d].assign(n3, 0.0);
    }
#pragma omp parallel for collapse(2)
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                long i = IDX(c, x, y, z);
                double ksq = ksq_of(c, x, y, z);
                if (ksq > MACH_EPSILON) {
                    gp[0][i] = -cplx(0.0, Kx(c, x)) * dh[i] / ksq;
                    gp[1][i] = -cplx(0.0, Kx(c, y)) * dh[i] / ksq;
                    gp[2][i] = -cplx(0.0, Kx(c, z)) * dh[i] / ksq;
                } else {
                    for (int d = 0; d < 3; ++d) { gp[d][i] = 0.0; uh[d][i] = 0.0; }
                }
            }
    RV g(n3);
    for (int d = 0; d < 3; ++d) {
        fftbwd(c, gp[d].data());
        real_part(c, gp[d], g.data());
        fftbwd(c, uh[d].data());
        real_part(c, uh[d], f + d * n3);
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) f[d * n3 + i] -= g[i];
    }
}

// HilbertGradient (3583-3627)
void hilbert(orc_ctx* c, double* g, double order) {
    const int n = c->n;
    for (int d = 0; d < 3; ++d) {
        CV a = to_complex(c, g + d * c->n3);
        fftfwd(c, a.data());
#pragma omp parallel for collapse(2)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    double ks = std::sqrt(ksq_of(c, x, y, z));
                    a[IDX(c, x, y, z)] /= (1.0 + std::pow(c->p.lambda1 * ks, 2.0 * order));
                }
        fftbwd(c, a.data());
        real_part(c, a, g + d * c->n3);
    }
}

// calc0thFourierModes (3048-3094): unnormalised k=0 coefficient
void zeroth_modes(orc_ctx* c, const double* u, double out[3]) {
    for (int d = 0; d < 3; ++d) {
        CV a = to_complex(c, u + d * c->n3);
        fftfwd(c, a.data());
        out[d] = a[0].real();
    }
}

// calcConstraintDerivativeL2 (984-1006)
void normal_l2(orc_ctx* c, const double* u, double* out) {
    const long n3 = c->n3;
    const double q = c->p.q;
    double nrm = lq_norm(c, u);
    RV a(n3);
    calc_uk(c, u, q - 2.0, a.data());
    for (int d = 0; d < 3; ++d) {
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) out[d * n3 + i] = a[i] * u[d * n3 + i];
        if (c->p.to_dealias && (q - 2.0 > MACH_EPSILON)) dealias_scalar(c, out + d * n3, 2.0);
    }
    const double f = std::pow(nrm, 1.0 - q);
    #pragma omp parallel for
    for (long i = 0; i < 3 * n3; ++i) out[i] = f * out[i];
}

// vectorTransport (1716-1768)
void vector_transport(orc_ctx* c, const double* u, double q, double B, const double* eta,
                      const double* xi, double* out) {
    const long n3 = c->n3, m = 3 * n3;
    RV w(m), a(n3), aux(m);
    #pragma omp parallel for
    for (long i = 0; i < m; ++i) w[i] = u[i] + eta[i];
    calc_uk(c, w.data(), q - 2.0, a.data());
    for (int d = 0; d < 3; ++d) {
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) aux[d * n3 + i] = a[i] * w[d * n3 + i];
        if (c->p.to_dealias && (q - 2.0 > MACH_EPSILON)) dealias_scalar(c, aux.data() + d * n3, 2.0);
    }
    double ir = field_inner(c, aux.data(), xi, 0);
    double ln = lq_norm(c, w.data());
    #pragma omp parallel for
    for (long i = 0; i < m; ++i) out[i] = xi[i] - std::pow(ln, -q) * ir * w[i];
    #pragma omp parallel for
    for (long i = 0; i < m; ++i) out[i] = B / ln * out[i];
}

// GradL2ForLq (1066-1211).  Temporaries are scoped so that each is freed
// once its last use is done (the reference holds all of them: 1076-1077);
// the arithmetic of every value is unchanged, which keeps 512^3 within a few
// tens of GB of host memory.
void grad_l2(orc_ctx* c, const double* u, double* v) {
    const long n3 = c->n3, m = 3 * n3;
    const double q = c->p.q, nu = c->p.visc, vc = c->p.visc_coef, pc = c->p.press_coef;
    RV a_q2(n3);
    calc_uk(c, u, q - 2.0, a_q2.data());
    RV gradP(m), dU(m), a3v(m);
    {
        RV aux(n3), tmp(n3), p(n3);
        nabla_u_nabla_ut(c, u, aux.data());
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) tmp[i] = -aux[i];
        solve_poisson(c, tmp.data(), 1.0, p.data());
        gradient(c, p.data(), gradP.data());
    }
    std::memcpy(dU.data(), u, sizeof(double) * m);
    laplacian(c, dU.data());
    {
        RV aux2(n3, 0.0);
        if (c->p.use_e_u) {
            RV e(m);
            unit_vector(c, u, e.data());
            for (int d = 0; d < 3; ++d)
                #pragma omp parallel for
                for (long i = 0; i < n3; ++i)
                    aux2[i] = aux2[i] + e[d * n3 + i] * (vc * nu * dU[d * n3 + i] - pc * gradP[d * n3 + i]);
            if (c->p.to_dealias && c->p.dealias_e_u) dealias_scalar(c, aux2.data(), 2.0);
            #pragma omp parallel for
            for (long i = 0; i < n3; ++i) aux2[i] = a_q2[i] * aux2[i];
            maybe_dealias(c, aux2.data(), 2.0);
            for (int d = 0; d < 3; ++d) {
                #pragma omp parallel for
                for (long i = 0; i < n3; ++i) a3v[d * n3 + i] = aux2[i] * e[d * n3 + i];
                if (c->p.to_dealias && c->p.dealias_e_u) dealias_scalar(c, a3v.data() + d * n3, 2.0);
            }
        } else {
            for (int d = 0; d < 3; ++d)
                #pragma omp parallel for
                for (long i = 0; i < n3; ++i)
                    aux2[i] = aux2[i] + u[d * n3 + i] * (vc * nu * dU[d * n3 + i] - pc * gradP[d * n3 + i]);
            maybe_dealias(c, aux2.data(), 2.0);
            {
                RV a_q4(n3);
                calc_uk(c, u, q - 4.0, a_q4.data());
                #pragma omp parallel for
                for (long i = 0; i < n3; ++i) aux2[i] = a_q4[i] * aux2[i];
            }
            maybe_dealias(c, aux2.data(), 2.0);
            for (int d = 0; d < 3; ++d) {
                #pragma omp parallel for
                for (long i = 0; i < n3; ++i) a3v[d * n3 + i] = aux2[i] * u[d * n3 + i];
                maybe_dealias(c, a3v.data() + d * n3, 2.0);
            }
        }
    }
    RV uq2u(m);
    for (int d = 0; d < 3; ++d) {
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) uq2u[d * n3 + i] = a_q2[i] * u[d * n3 + i];
        maybe_dealias(c, uq2u.data() + d * n3, 2.0);
    }
    RV a4v(m);
    {
        RV aux3(n3), aux4(n3);
        divergence(c, uq2u.data(), aux3.data());
        solve_poisson(c, aux3.data(), 1.0, aux4.data());
        gradient(c, aux4.data(), a4v.data());
    }
    RV a5v(m);
    {
        RV gU = grad_tensor(c, u);  // gU[k][i] = d_i u_k  (gradUk(:,:,:,ii))
        for (int ii = 0; ii < 3; ++ii) {
            #pragma omp parallel for
            for (long i = 0; i < n3; ++i)
                a5v[ii * n3 + i] = GU(gU, c, 0, ii)[i] * a4v[0 * n3 + i] + GU(gU, c, 1, ii)[i] * a4v[1 * n3 + i] +
                                   GU(gU, c, 2, ii)[i] * a4v[2 * n3 + i];
            maybe_dealias(c, a5v.data() + ii * n3, 2.0);
        }
    }
    laplacian(c, uq2u.data());  // the a7v term: uq2u is not read again
    const double* a7v = uq2u.data();
    RV a6(n3);
    for (int d = 0; d < 3; ++d) {
        double* a4 = a4v.data() + d * n3;
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) a4[i] = a_q2[i] * gradP[d * n3 + i];
        maybe_dealias(c, a4, 2.0);
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i) a6[i] = a_q2[i] * dU[d * n3 + i];
        maybe_dealias(c, a6.data(), 2.0);
        #pragma omp parallel for
        for (long i = 0; i < n3; ++i)
            v[d * n3 + i] = (q - 2.0) * a3v[d * n3 + i] - pc * a4[i] + pc * 2.0 * a5v[d * n3 + i] +
                            vc * nu * a6[i] + vc * nu * a7v[d * n3 + i];
    }
}

// eval_J (optimization.f90:520-547)
double eval_J(orc_ctx* c, const double* field, int mode) {
    const long m = 3 * c->n3;
    RV aux(field, field + m);
    double out[3];
    switch (mode) {
        case 0:
            R_parts(c, aux.data(), out);
            return out[0];
        case 1:
            c->n_evals++;
            rescale(c, aux.data(), c->p.B);
            R_parts(c, aux.data(), out);
            return -1.0 * out[0];
        case 2:
            return lq_norm(c, aux.data());
    }
    return 0.0;
}

double lm_eval(orc_ctx* c, const double* phi, const double* d, double t, RV& buf) {
    const long m = 3 * c->n3;
    #pragma omp parallel for
    for (long i = 0; i < m; ++i) buf[i] = phi[i] + t * d[i];
    return eval_J(c, buf.data(), 1);
}

// mnbrak (optimization.f90:613-778) without the save_linemin_data I/O.
// Returns 0 ok; flag as the reference (1 uphill, 2 ITMAX).
int mnbrak(orc_ctx* c, const double* phi, const double* grad, double tA0, double tB0, double tau_brack[2],
           int* myflag) {
    const double GOLD = (1.0 + std::sqrt(5.0)) / 2.0;
    const double CGOLD = 1.0 / GOLD;
    const double GLIMIT = 10.0;
    const int ITMAX = 100;
    RV buf(3 * c->n3);
    double tA = tA0, tB = std::max(tB0, MACH_EPSILON), tC = 0.0, tP, FP, Pmax, R, Q;
    double FA = lm_eval(c, phi, grad, tA, buf);
    double FB = lm_eval(c, phi, grad, tB, buf);
    double FC = 0.0;
    int brakIter = 0;
    while (FB > FA && tB > MACH_EPSILON) {
        tB = CGOLD * tB;
        FB = lm_eval(c, phi, grad, tB, buf);
    }
    if (tB <= MACH_EPSILON) {
        *myflag = 1;
        return 1;
    }
    tC = GOLD * tB;
    FC = lm_eval(c, phi, grad, tC, buf);
    while (FB >= FC && brakIter < ITMAX) {
        brakIter++;
        tC = GOLD * tC;
        FC = lm_eval(c, phi, grad, tC, buf);
        R = (tB - tA) * (FB - FC);
        Q = (tB - tC) * (FB - FA);
        tP = tB - 0.5 * ((tB - tC) * Q - (tB - tA) * R) / std::copysign(std::max(std::fabs(Q - R), MACH_EPSILON), Q - R);
        Pmax = tB + GLIMIT * (tC - tB);
        if ((tB - tP) * (tP - tC) > 0) {
            FP = lm_eval(c, phi, grad, tP, buf);
            if (FP < FC) {
                tA = tB; FA = FB; tB = tP; FB = FP;
                break;
            } else if (FP > FB) {
                tC = tP; FC = FP;
                break;
            }
            tP = tC + GOLD * (tC - tB);
            FP = lm_eval(c, phi, grad, tP, buf);
        } else if ((tC - tP) * (tP - Pmax) > 0) {
            FP = lm_eval(c, phi, grad, tP, buf);
            if (FP < FC) {
                tB = tC; tC = tP; FB = FC; FC = FP;
                tP = tC + GOLD * (tC - tB);
                FP = lm_eval(c, phi, grad, tP, buf);
            }
        } else if ((tP - Pmax) * (Pmax - tC) >= 0) {
            tP = Pmax;
            FP = lm_eval(c, phi, grad, tP, buf);
        } else {
            tP = tC + GOLD * (tC - tB);
            FP = lm_eval(c, phi, grad, tP, buf);
        }
        tA = tB; tB = tC; tC = tP;
        FA = FB; FB = FC; FC = FP;
    }
    tau_brack[0] = tA;
    tau_brack[1] = tC;
    *myflag = brakIter >= ITMAX ? 2 : 0;
    return *myflag;
}

// brent (optimization.f90:784-951) without the brent-info file I/O.  The
// constants are Fortran default-real literals widened to double (804-806).
double brent(orc_ctx* c, const double* phi, const double* grad, const double tau_brack[2]) {
    const int ITMAX = 300;
    const double TOL = (double)1E-6f;
    const double ZEPS = (double)1E-8f;
    const double CGOLD = (double).381966f;
    RV buf(3 * c->n3);
    double D = 0.0, A = std::min(tau_brack[0], tau_brack[1]), B = std::max(tau_brack[0], tau_brack[1]);
    double V = tau_brack[1] * CGOLD, W = V, X = V, E = 0.0, ETEMP, P, Q, R, U, XM, TOL1, TOL2;
    double FX = lm_eval(c, phi, grad, D, buf);  // logged value at tau = 0 (833-834)
    FX = lm_eval(c, phi, grad, X, buf);
    double FV = FX, FW = FX, FU;
    for (int j = 1; j <= ITMAX; ++j) {
        XM = 0.5 * (A + B);
        TOL1 = TOL * std::fabs(X) + ZEPS;
        TOL2 = 2.0 * TOL1;
        if (std::fabs(X - XM) <= (TOL2 - 0.5 * (B - A))) break;
        int FLAG = 1;
        if (std::fabs(E) > TOL1) {
            R = (X - W) * (FX - FV);
            Q = (X - V) * (FX - FW);
            P = (X - V) * Q - (X - W) * R;
            Q = 2.0 * (Q - R);
            if (Q > 0.0) P = -P;
            Q = std::fabs(Q);
            ETEMP = E;
            E = D;
            if ((std::fabs(P) >= std::fabs(0.5 * Q * ETEMP)) || (P <= Q * (A - X)) || (P >= Q * (B - X)))
                FLAG = 1;
            else
                FLAG = 2;
        }
        if (FLAG == 1) {
            E = (X >= XM) ? A - X : B - X;
            D = CGOLD * E;
        } else {
            D = P / Q;
            U = X + D;
            if ((U - A < TOL2) || (B - U < TOL2)) D = std::copysign(TOL1, XM - X);
        }
        U = (std::fabs(D) >= TOL1) ? X + D : X + std::copysign(TOL1, D);
        FU = lm_eval(c, phi, grad, U, buf);
        if (FU <= FX) {
            if (U >= X) A = X; else B = X;
            V = W; FV = FW; W = X; FW = FX; X = U; FX = FU;
        } else {
            if (U < X) A = U; else B = U;
            if ((FU <= FW) || (W == X)) {
                V = W; FV = FW; W = U; FW = FU;
            } else if ((FU <= FV) || (V == X) || (V == W)) {
                V = U; FV = FU;
            }
        }
    }
    return X;
}

}  // namespace

// ---------------------------------------------------------------------------
// Diagnostics the reference computes around the CG loop (maxdLpdt.f90:263-299,
// optimization.f90:119-123, 377-384)
// ---------------------------------------------------------------------------

// calculate_spectral_data (function_ops.f90:2614-2677): shell sums of
// |fftfwd(u_c)|^2 over kk_min < |K| <= kk_max, kk = 2 pi i, i = 0..n-1, then
// (normalizeSpectrumByL2Norm, global_variables.f90:76) scaled by
// <u,u>_L2 / (2 pi sum).  out[0..n) = kk_max, out[n..2n) = the spectrum.
void spectral_data(orc_ctx* c, const double* u, double* out, int normalize) {
    const int n = c->n;
    const long n3 = c->n3;
    std::vector<CV> fu(3);
    for (int d = 0; d < 3; ++d) {
        fu[d] = to_complex(c, u + d * n3);
        fftfwd(c, fu[d].data());
    }
    for (int i = 0; i < n; ++i) {
        const double kk_min = 2.0 * c->PI * (double)i;
        const double kk_max = 2.0 * c->PI * (double)(i + 1);
        out[i] = kk_max;
        double s = 0.0;
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const double nk = std::sqrt(Kx(c, x) * Kx(c, x) + Kx(c, y) * Kx(c, y) + Kx(c, z) * Kx(c, z));
                    if (kk_min < nk && nk <= kk_max) {
                        const long j = IDX(c, x, y, z);
                        s += std::norm(fu[0][j]) + std::norm(fu[1][j]) + std::norm(fu[2][j]);
                    }
                }
        out[n + i] = s;
    }
    if (normalize) {
        double l2 = 0.0;
        for (int d = 0; d < 3; ++d) l2 += inner_l2(c, u + d * n3, u + d * n3);
        double tot = 0.0;
        for (int i = 0; i < n; ++i) tot += out[n + i];
        const double spectral_Ener = 2.0 * c->PI * tot;
        for (int i = 0; i < n; ++i) out[n + i] = l2 / spectral_Ener * out[n + i];
    }
}

// vel2vort + Enstrophy + calc_global_summed_enstrophy (function_ops.f90:
// 2422-2467): 1/2 ||curl u||^2 summed over the components
double summed_enstrophy(orc_ctx* c, const double* u) {
    const int n = c->n;
    const long n3 = c->n3;
    CV uh[3];
    for (int d = 0; d < 3; ++d) {
        uh[d] = to_complex(c, u + d * n3);
        fftfwd(c, uh[d].data());
    }
    double ens[3] = {0.0, 0.0, 0.0};
    CV w(n3);
    RV wr(n3);
    for (int d = 0; d < 3; ++d) {
#pragma omp parallel for collapse(2)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const long i = IDX(c, x, y, z);
                    const cplx ik1(0.0, Kx(c, x)), ik2(0.0, Kx(c, y)), ik3(0.0, Kx(c, z));
                    if (d == 0) w[i] = ik2 * uh[2][i] - ik3 * uh[1][i];
                    if (d == 1) w[i] = ik3 * uh[0][i] - ik1 * uh[2][i];
                    if (d == 2) w[i] = ik1 * uh[1][i] - ik2 * uh[0][i];
                }
        CV a = w;
        fftbwd(c, a.data());
        real_part(c, a, wr.data());
        for (long i = 0; i < n3; ++i) ens[d] = ens[d] + 0.5 * wr[i] * wr[i] * c->dV;
    }
    return ens[0] + ens[1] + ens[2];
}

// calc_global_dEnstrophydt (function_ops.f90:1417-1481): out = {R1 + R2, R1, R2},
// R1 = -viscCoefficient visc ||Lap u||^2, R2 = <P2((u.grad) u), Lap u>
void dEnstrophydt(orc_ctx* c, const double* u, double out[3]) {
    const long n3 = c->n3, m = 3 * n3;
    RV lap(u, u + m);
    laplacian(c, lap.data());
    const double R1 = -c->p.visc_coef * c->p.visc * field_inner(c, lap.data(), lap.data(), 0);
    RV gU = grad_tensor(c, u);  // gU[i][j] = d_j u_i
    RV ug(m, 0.0);
    for (int ii = 0; ii < 3; ++ii)
        for (int jj = 0; jj < 3; ++jj)
#pragma omp parallel for
            for (long i = 0; i < n3; ++i) ug[ii * n3 + i] = ug[ii * n3 + i] + u[jj * n3 + i] * GU(gU, c, ii, jj)[i];
    for (int ii = 0; ii < 3; ++ii) maybe_dealias(c, ug.data() + ii * n3, 2.0);
    const double R2 = field_inner(c, ug.data(), lap.data(), 0);
    out[0] = R1 + R2;
    out[1] = R1;
    out[2] = R2;
}

// calc_uv_scalar (function_ops.f90:2069-2081)
void uv_scalar(orc_ctx* c, const double* a, const double* b, double* res) {
#pragma omp parallel for
    for (long i = 0; i < c->n3; ++i) res[i] = a[i] * b[i];
    maybe_dealias(c, res, 2.0);
}

// calc_local_pointwise_dLqdt_inclParts (function_ops.f90:1224-1291): the
// fields R1 + R2 + R3, R1 + R2 and R3 (res is 3 n^3)
void pointwise_R(orc_ctx* c, const double* u, double* res) {
    const long n3 = c->n3;
    const double q = c->p.q, nu = c->p.visc, vc = c->p.visc_coef, pc = c->p.press_coef;
    RV a_q2(n3), aux(n3), e(3 * n3), a_q4(n3), p(n3), tmp(n3), pt(n3), R1(n3), R2(n3), R3(n3);
    calc_uk(c, u, q - 2.0, a_q2.data());
    nabla_mod_squared(c, u, aux.data());
    uv_scalar(c, a_q2.data(), aux.data(), pt.data());
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) R1[i] = -vc * nu * pt[i];
    unit_vector(c, u, e.data());
    if (c->p.use_e_u) {
        vgraduvgradu(c, u, e.data(), aux.data());
        uv_scalar(c, a_q2.data(), aux.data(), pt.data());
    } else {
        calc_uk(c, u, q - 4.0, a_q4.data());
        vgraduvgradu(c, u, u, aux.data());
        uv_scalar(c, a_q4.data(), aux.data(), pt.data());
    }
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) R2[i] = -vc * (q - 2.0) * nu * pt[i];
    nabla_u_nabla_ut(c, u, aux.data());
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) tmp[i] = -aux[i];
    solve_poisson(c, tmp.data(), 1.0, p.data());
    const double* mult = c->p.use_e_u ? a_q2.data() : a_q4.data();
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) aux[i] = p[i] * mult[i];
    maybe_dealias(c, aux.data(), 2.0);
    vvgradu(c, u, c->p.use_e_u ? e.data() : u, tmp.data());
    uv_scalar(c, aux.data(), tmp.data(), pt.data());
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) R3[i] = pc * (q - 2.0) * pt[i];
#pragma omp parallel for
    for (long i = 0; i < n3; ++i) {
        res[i] = R1[i] + R2[i] + R3[i];
        res[n3 + i] = R1[i] + R2[i];
        res[2 * n3 + i] = R3[i];
    }
}

// ---- kappa_test_pert (function_ops.f90:615-977) ---------------------------
namespace {

// The random fields of create-random-poly-b and save-random are drawn from
// Fortran's unseeded random_number there (784-785, 937-938); here from a
// seeded counter generator (splitmix64 finaliser of seed + (i+1) * golden
// gamma, top 53 bits), element i in the array order of phi_pert(x,y,z,c).
double pert_uniform(unsigned long long seed, long i) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// faux(:,:,:,ll) *= f(norm_K), 0 where norm_K < MACH_EPSILON, through one
// fftfwdv / fftbwdv round trip per component (e.g. 771-793)
template <class F>
void pert_filter(orc_ctx* c, double* phi, F f) {
    const int n = c->n;
    for (int d = 0; d < 3; ++d) {
        CV a = to_complex(c, phi + d * c->n3);
        fftfwd(c, a.data());
#pragma omp parallel for collapse(2)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const long i = IDX(c, x, y, z);
                    const double norm_K = std::sqrt(Kx(c, x) * Kx(c, x) + Kx(c, y) * Kx(c, y) + Kx(c, z) * Kx(c, z));
                    if (norm_K < MACH_EPSILON)
                        a[i] = 0.0;
                    else
                        a[i] *= f(norm_K);
                }
        fftbwd(c, a.data());
        real_part(c, a, phi + d * c->n3);
    }
}

// returns 1 when successful (the reference's `successful`), 0 when a load-*
// type had no field (in == nullptr: phi taken as 0), -1 for an unknown type
int kappa_pert(orc_ctx* c, const char* type, double m1, double m2, double m3, const double* in,
               unsigned long long seed, double* phi) {
    const int n = c->n;
    const long n3 = c->n3;
    const std::string t(type);
    const double PI = c->PI;
    int ok = 1;
    auto load = [&] {
        if (in) {
            std::memcpy(phi, in, sizeof(double) * 3 * n3);
        } else {
            std::memset(phi, 0, sizeof(double) * 3 * n3);
            ok = 0;
        }
    };
    auto poly = [&](double nk) { return std::pow(10.0, m2) * std::pow(nk / ((double)n / 4.0), m1); };
    auto random_field = [&] {
        // random_number, 2 phi - 1, the k = 0 mode removed, divAvg_free, and
        // phi / (100 <phi, phi>_L2) (784-803, 937-956)
        for (long i = 0; i < 3 * n3; ++i) phi[i] = 2.0 * pert_uniform(seed, i) - 1.0;
        pert_filter(c, phi, [](double) { return 1.0; });
        divavg_free(c, phi);
        const double normalization_const = 100.0 * field_inner(c, phi, phi, 0);
        for (long i = 0; i < 3 * n3; ++i) phi[i] = phi[i] / normalization_const;
    };
    const double dx = 1.0 / (double)n;
    if (t == "sine" || t == "divfree-sine") {  // 658-688
        const bool df = t == "divfree-sine";
        const double m2e = df ? m1 + m3 : m2;
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const double X = (double)x * dx, Y = (double)y * dx, Z = (double)z * dx;
                    const long i = IDX(c, x, y, z);
                    phi[i] = std::sin(2.0 * PI * m1 * X) * std::cos(2.0 * PI * m2e * Y) * std::cos(2.0 * PI * m3 * Z);
                    phi[n3 + i] =
                        -std::cos(2.0 * PI * m1 * X) * std::sin(2.0 * PI * m2e * Y) * std::cos(2.0 * PI * m3 * Z);
                    phi[2 * n3 + i] =
                        std::cos(2.0 * PI * m1 * X) * std::cos(2.0 * PI * m2e * Y) * std::sin(2.0 * PI * m3 * Z);
                }
        if (!df) divavg_free(c, phi);
    } else if (t == "load-te0080") {  // 652-655
        load();
    } else if (t == "load-random-a" || t == "load-random-b") {  // 691-701
        load();
        divavg_free(c, phi);
    } else if (t == "load-random-smooth-a" || t == "load-random-smooth-b") {  // 703-711, 923-930
        load();
        for (int d = 0; d < 3; ++d) dealias_scalar(c, phi + d * n3, 20.0);
        if (t == "load-random-smooth-a") divavg_free(c, phi);
    } else if (t == "load-k-random-a" || t == "load-k-random-b") {  // 713-765
        load();
        pert_filter(c, phi, [&](double) { return m1; });
        divavg_free(c, phi);
    } else if (t == "load-random-poly-a" || t == "load-random-poly-b") {  // 768-792, 830-854
        load();
        pert_filter(c, phi, poly);
        divavg_free(c, phi);
    } else if (t == "load-random-exp-a" || t == "load-random-exp-b") {  // 857-920
        load();
        pert_filter(c, phi, [](double nk) { return std::pow(10.0, -nk / 5.0); });
        divavg_free(c, phi);
    } else if (t == "create-random-poly-b") {  // 795-827
        random_field();
        pert_filter(c, phi, poly);
        divavg_free(c, phi);
    } else if (t == "save-random") {  // 932-956 (the field written to n<NNNN>_random.nc)
        random_field();
    } else {
        return -1;
    }
    return ok;
}

}  // namespace

extern "C" {

void orc_default_params(orc_params* p, int n, double q, double B) {
    p->n = n;
    p->q = q;
    p->B = B;
    p->visc = 1.0;
    p->lambda1 = 0.1;
    p->visc_coef = 1.0;
    p->press_coef = 1.0;
    p->to_dealias = 1;
    // set_e_u_or_just_u with use_e_u_auto_for_q_less_4 (initialize.f90:75-86)
    p->use_e_u = (q < 4.0 - MACH_EPSILON) ? 1 : 0;
    p->dealias_e_u = 1;
    p->threads = 0;
}

orc_ctx* orc_create(const orc_params* p) {
    orc_ctx* c = new orc_ctx;
    c->p = *p;
    c->n = p->n;
    c->n3 = (long)p->n * p->n * p->n;
    c->dV = 1.0 / ((double)p->n * (double)p->n * (double)p->n);  // initialize.f90:162
    c->PI = 4.0 * std::atan2(1.0, 1.0);                          // initialize.f90:164
    c->K.resize(p->n);
    for (int i = 0; i < p->n; ++i)
        c->K[i] = (i <= p->n / 2) ? 2.0 * c->PI * (double)i : 2.0 * c->PI * (double)(i - p->n);
    c->fft.init(p->n);
#ifdef _OPENMP
    if (p->threads > 0) omp_set_num_threads(p->threads);
#endif
    return c;
}

void orc_destroy(orc_ctx* c) { delete c; }
int orc_eval_count(orc_ctx* c) { return c->n_evals; }

void orc_fft_c2c(orc_ctx* c, double* data, int dir) {
    cplx* a = reinterpret_cast<cplx*>(data);
    if (dir < 0) fftfwd(c, a); else fftbwd(c, a);
}

void orc_dealias_scalar(orc_ctx* c, double* g, double order) { dealias_scalar(c, g, order); }
void orc_gradient(orc_ctx* c, const double* u, double* grad) { gradient(c, u, grad); }
void orc_divergence(orc_ctx* c, const double* u, double* div) { divergence(c, u, div); }
void orc_laplacian(orc_ctx* c, double* f) { laplacian(c, f); }
void orc_solve_poisson(orc_ctx* c, const double* f, double l, double* phi) { solve_poisson(c, f, l, phi); }
void orc_calc_uk(orc_ctx* c, const double* u, double k, double* uk) { calc_uk(c, u, k, uk); }
void orc_unit_vector(orc_ctx* c, const double* u, double* e) { unit_vector(c, u, e); }
void orc_divavg_free(orc_ctx* c, double* u) { divavg_free(c, u); }
void orc_hilbert_gradient(orc_ctx* c, double* g, double order) { hilbert(c, g, order); }
double orc_inner_product(orc_ctx* c, const double* f, const double* g, int htype) { return inner(c, f, g, htype); }
double orc_field_inner(orc_ctx* c, const double* f, const double* g, int htype) { return field_inner(c, f, g, htype); }
void orc_zeroth_modes(orc_ctx* c, const double* u, double out[3]) { zeroth_modes(c, u, out); }
double orc_lq_norm(orc_ctx* c, const double* u) { return lq_norm(c, u); }
void orc_rescale(orc_ctx* c, double* u, double B) { rescale(c, u, B); }
void orc_normal_l2(orc_ctx* c, const double* u, double* out) { normal_l2(c, u, out); }
void orc_vector_transport(orc_ctx* c, const double* u, double q, double B, const double* eta, const double* xi,
                          double* out) {
    vector_transport(c, u, q, B, eta, xi, out);
}
void orc_R_parts(orc_ctx* c, const double* u, double out[3]) { R_parts(c, u, out); }
void orc_grad_l2(orc_ctx* c, const double* u, double* v) { grad_l2(c, u, v); }
double orc_eval_J(orc_ctx* c, const double* u, int mode) { return eval_J(c, u, mode); }
void orc_spectral_data(orc_ctx* c, const double* u, double* out, int normalize) {
    spectral_data(c, u, out, normalize);
}
double orc_summed_enstrophy(orc_ctx* c, const double* u) { return summed_enstrophy(c, u); }
void orc_dEnstrophydt(orc_ctx* c, const double* u, double out[3]) { dEnstrophydt(c, u, out); }
void orc_pointwise_R(orc_ctx* c, const double* u, double* res) { pointwise_R(c, u, res); }
int orc_kappa_pert(orc_ctx* c, const char* type, double m1, double m2, double m3, const double* in,
                   unsigned long long seed, double* out) {
    return kappa_pert(c, type, m1, m2, m3, in, seed, out);
}
int orc_mnbrak(orc_ctx* c, const double* phi, const double* d, double tA0, double tB0, double tau_brack[2],
               int* flag) {
    *flag = 0;
    return mnbrak(c, phi, d, tA0, tB0, tau_brack, flag);
}
double orc_brent(orc_ctx* c, const double* phi, const double* d, const double tau_brack[2]) {
    return brent(c, phi, d, tau_brack);
}

// maxdLqdt (optimization.f90:7-514), flags at their defaults
// (useTangentialGradient, useConjugateGradient, useRiemannianGeometry,
// normalizeGradient all true; kappaTest off; no file output).
int orc_maxdlqdt(orc_ctx* c, double* uvec, int max_iter, double optim_tol, int start_iter, orc_iter_cb cb,
                 void* user, int* flag) {
    const long n3 = c->n3, m = 3 * n3;
    const double q = c->p.q, Bc = c->p.B;
    const int resetEvery = 25, rollSize = 10;
    RV gradJ1(m), gradJproj(m), normalL2(m), normalHs(m), gu0(m, 0.0), gu1(m), d0(m, 0.0), d1(m), vtg0(m, 0.0),
        vtd0(m, 0.0), tmp(m), tmp2(m);
    *flag = 0;
    rescale(c, uvec, Bc);          // 61
    divavg_free(c, uvec);          // 62
    double J0 = eval_J(c, uvec, 0);  // 78
    double J1 = J0, deltaJ;
    int iter = start_iter;
    double tau0 = std::pow(10.0, 2.0), tau1 = tau0;
    std::vector<double> roll(rollSize, 0.0);
    double avgImp = 1.0;
    int while_flag = 0;
    double tau_brack[2] = {0.0, 0.0};
    while (std::fabs(avgImp) > optim_tol && iter < max_iter && while_flag < 1) {
        iter++;
        int ev0 = c->n_evals;
        grad_l2(c, uvec, gradJ1.data());                       // 146
        const double s = (3.0 / 2.0) - (1.0 / q);              // 150
        hilbert(c, gradJ1.data(), s);                          // 151
        divavg_free(c, gradJ1.data());                         // 153
        normal_l2(c, uvec, normalL2.data());                   // 162
        normalHs = normalL2;
        hilbert(c, normalHs.data(), s);                        // 164
        divavg_free(c, normalHs.data());                       // 169
        double alpha = field_inner(c, normalHs.data(), gradJ1.data(), 1);
        alpha = alpha / field_inner(c, normalHs.data(), normalHs.data(), 1);  // 170-171
        #pragma omp parallel for
        for (long i = 0; i < m; ++i) gradJproj[i] = gradJ1[i] - alpha * normalHs[i];  // 177
        gu1 = gradJproj;                                                             // 202
        {
            double r = std::sqrt(field_inner(c, uvec, uvec, 1) / field_inner(c, gu1.data(), gu1.data(), 1));
            #pragma omp parallel for
            for (long i = 0; i < m; ++i) gu1[i] = r * gu1[i];  // 213
        }
        #pragma omp parallel for
        for (long i = 0; i < m; ++i) tmp[i] = gu1[i] - vtg0[i];
        double beta = field_inner(c, gu1.data(), tmp.data(), 1);       // 226
        double g0n = field_inner(c, gu0.data(), gu0.data(), 1);        // 227
        if (g0n < MACH_EPSILON || beta < MACH_EPSILON) beta = 0.0; else beta = beta / g0n;
        if (iter % resetEvery == 0) beta = 0.0;                        // 235-238
        #pragma omp parallel for
        for (long i = 0; i < m; ++i) d1[i] = gu1[i] + beta * vtd0[i];  // 240
        double nG = std::sqrt(field_inner(c, gu1.data(), gu1.data(), 1));
        double nT = std::sqrt(field_inner(c, vtd0.data(), vtd0.data(), 1));
        double nD = std::sqrt(field_inner(c, d1.data(), d1.data(), 1));
        int mflag = 0;
        mnbrak(c, uvec, d1.data(), 0.0, tau0, tau_brack, &mflag);      // 269
        if (mflag != 0) {
            *flag = mflag;
            if (cb) {
                orc_iter_info info = {};
                info.iter = iter; info.J0 = J0; info.mnbrak_flag = mflag; info.beta = beta;
                info.n_evals = c->n_evals - ev0;
                cb(&info, user);
            }
            while_flag = 1;
            break;
        }
        tau1 = brent(c, uvec, d1.data(), tau_brack);  // 297
        if (tau1 > TAU_MAX) {                          // 310-314
            while_flag = 1;
            *flag = 4;
            tau1 = 0.0;
        }
        #pragma omp parallel for
        for (long i = 0; i < m; ++i) tmp2[i] = tau1 * d1[i];
        vector_transport(c, uvec, q, Bc, tmp2.data(), gu1.data(), vtg0.data());  // 326
        vector_transport(c, uvec, q, Bc, tmp2.data(), d1.data(), vtd0.data());   // 327
        #pragma omp parallel for
        for (long i = 0; i < m; ++i) uvec[i] = uvec[i] + tau1 * d1[i];           // 345
        rescale(c, uvec, Bc);                                                   // 346
        J1 = eval_J(c, uvec, 0);                                                // 349
        deltaJ = (J1 - J0) / std::fabs(J0);
        orc_iter_info info = {};
        info.iter = iter; info.tau_a = tau_brack[0]; info.tau = tau1; info.tau_b = tau_brack[1];
        info.J0 = J0; info.deltaJ = deltaJ; info.J1 = J1; info.beta = beta; info.alpha = alpha;
        info.norm_grad = nG; info.norm_td0 = nT; info.norm_d1 = nD;
        info.n_evals = c->n_evals - ev0; info.mnbrak_flag = 0;
        if (deltaJ < -MACH_EPSILON) {  // 351-366
            *flag = 5;
            if (cb) cb(&info, user);
            while_flag = 1;
            break;
        }
        info.u_norm_q = lq_norm(c, uvec);  // 421
        {
            double parts[3];
            R_parts(c, uvec, parts);  // 423
            info.R = parts[0]; info.R12 = parts[1]; info.R3 = parts[2];
        }
        if (cb) cb(&info, user);
        J0 = J1;      // 432
        gu0 = gu1;    // 434
        tau0 = tau1;  // 435
        d0 = d1;      // 436
        for (int i = rollSize - 1; i >= 1; --i) roll[i] = roll[i - 1];  // 439
        roll[0] = deltaJ;                                               // 443
        double ssum = 0.0;
        for (int i = 0; i < rollSize; ++i) ssum += roll[i];
        avgImp = ssum / (double)(iter - start_iter);  // 445
    }
    return iter;
}

}  // extern "C"
