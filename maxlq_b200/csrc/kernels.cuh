// kernels.cuh -- the pass kernels of the pruned spectral pipeline.
//
// HBM layouts (T = float or double, cpx<T> interleaved):
//   phys  : T        [z][y][x]             N^3, x fastest (Fortran (n1,n2,n3))
//   xs    : cpx<T>   [z][y][kx]            after the x real FFT, kx < nx
//   ys    : cpx<T>   [z][ky'][kx]          after the y FFT, ky' < nb (band order)
//   spec  : cpx<T|double> [kz'][ky'][kx]   pruned Fourier coefficients (1/N^3)
// Forward pipeline : phys --x-stage(functor, r2c)--> xs --y fwd--> ys --z stage--> spec
// Inverse pipeline : spec --z stage--> ys --y inv--> xs --x inv (c2r)--> phys
// The z stage is where the whole wavevector is known: masks, derivative and
// Poisson symbols, Parseval reductions and spectral round trips live there.
#pragma once

#include "fft.cuh"

namespace mlq {

constexpr int MAX_ARR = 8;    // arrays per pass launch
constexpr int MAX_RED = 8;    // reduction slots per launch
constexpr int RED_THREADS = 256;

// ----------------------------------------------------------------------------
// Block reduction of NR doubles into partials[blockLinear*NR + r].
// ----------------------------------------------------------------------------
template <int NR>
__device__ __forceinline__ void block_reduce_store(const double* acc, double* partials, int block_lin) {
    __shared__ double red_smem[32][NR > 0 ? NR : 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double v = acc[r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red_smem[warp][r] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double v = lane < nw ? red_smem[lane][r] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) partials[(long)block_lin * NR + r] = v;
        }
    }
}

// results[dst + r] = scale * sum_b partials[b*nr + r]   (fixed order: deterministic)
static __global__ void finalize_partials_kernel(const double* __restrict__ partials, int nblocks, int nr, double scale,
                                         double* __restrict__ results, int dst, int accumulate) {
    __shared__ double sm[RED_THREADS];
    for (int r = 0; r < nr; ++r) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partials[(long)b * nr + r];
        sm[threadIdx.x] = v;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) results[dst + r] = (accumulate ? results[dst + r] : 0.0) + scale * sm[0];
        __syncthreads();
    }
}

// ----------------------------------------------------------------------------
// x stage, forward: functor on physical inputs, then real FFT along x.
// Each CTA owns `lx` consecutive (y,z) lines.
// ----------------------------------------------------------------------------
template <typename T>
struct XFwdArgs {
    int n, nx;          // grid, kept kx per output line
    int lx;             // lines per CTA
    const T* in[24];    // physical inputs
    cpx<T>* out[MAX_ARR];
    FftPlan plan_half;  // length n/2
    int tw_n_off;       // offset of W_n (length n) in the twiddle pool
    const cpx<double>* tw;
    double* partials;
    long nlines = 0;    // lines (rows along x) processed; a slab of planes is nlines = planes * n
    int px = 0;         // row pitch of the outputs in elements (0: nx); compile-time kernels only
    // Set to 1 when a forward transform meets a non-finite value (null: not
    // checked).  The DC bin of a packed line is the sum of all its values, so
    // it is non-finite exactly when some input of the line is (or the sum
    // overflows), the condition of the reference's NaN scan after fftfwd
    // (fftwfunction.f90:78-89).
    double* nanflag = nullptr;
};

template <typename T>
__device__ __forceinline__ bool cpx_finite(cpx<T> v) {
    return isfinite(v.x) && isfinite(v.y);
}

template <typename T, class F>
__global__ void __launch_bounds__(256) xfwd_kernel(XFwdArgs<T> a, F f) {
    constexpr int NIN = F::NIN, NOUT = F::NOUT, NR = F::NRED;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, h = n / 2, lx = a.lx;
    const int nl = NOUT * lx;  // FFT lines in this CTA
    cpx<T>* bufA = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* bufB = bufA + (long)h * nl;
    T* rA = reinterpret_cast<T*>(bufA);
    const long line0 = (long)blockIdx.x * lx;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;

    for (int p = threadIdx.x; p < lx * n; p += blockDim.x) {
        const int l = p / n, x = p - l * n;
        const long g = (line0 + l) * n + x;
        T vin[NIN];
#pragma unroll
        for (int i = 0; i < NIN; ++i) vin[i] = a.in[i][g];
        T vout[NOUT > 0 ? NOUT : 1];
        f(vin, vout, acc);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) rA[2 * ((long)(x >> 1) * nl + o * lx + l) + (x & 1)] = vout[o];
    }
    __syncthreads();
    cpx<T>* Z = fft_lines<-1, T>(bufA, bufB, a.plan_half, nl, nl, a.tw, threadIdx.x, blockDim.x);
    if (a.nanflag && (int)threadIdx.x < nl && !cpx_finite(Z[threadIdx.x])) *a.nanflag = 1.0;
    // split into the half spectrum of the real line: X[k] = E[k] + W_n^k O[k]
    const double2* twn = reinterpret_cast<const double2*>(a.tw + a.tw_n_off);
    for (int p = threadIdx.x; p < nl * a.nx; p += blockDim.x) {
        const int lo = p / a.nx, k = p - lo * a.nx;
        const int o = lo / lx, l = lo - o * lx;
        const cpx<T> zk = Z[(long)(k % h) * nl + lo];
        const cpx<T> zc = conj(Z[(long)((h - k) % h) * nl + lo]);
        const cpx<T> E = (zk + zc) * T(0.5);
        const cpx<T> D = (zk - zc) * T(0.5);
        const cpx<T> O = mk<T>(D.y, -D.x);  // -i * D
        const double2 w = __ldg(twn + k);   // exp(-2 pi i k / n)
        const cpx<T> X = E + O * mk<T>((T)w.x, (T)w.y);
        a.out[o][(line0 + l) * a.nx + k] = X;
    }
    if constexpr (NR > 0) block_reduce_store<NR>(acc, a.partials, blockIdx.x);
}

// ----------------------------------------------------------------------------
// Pointwise physical-space kernels: reduce-only (NOUT = 0) or map.
// ----------------------------------------------------------------------------
template <typename T>
struct PArgs {
    static constexpr int MAX_IN = 24, MAX_OUT = 14;
    long npts;
    const T* in[MAX_IN];
    T* out[MAX_OUT];
    double* partials;
};

template <typename T, class F>
__global__ void __launch_bounds__(RED_THREADS) pointwise_kernel(PArgs<T> a, F f) {
    constexpr int NIN = F::NIN, NOUT = F::NOUT, NR = F::NRED;
    using T2 = cpx<T>;  // two consecutive points per load and store
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    const long npairs = a.npts / 2;
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < npairs; g += (long)gridDim.x * blockDim.x) {
        T2 vin[NIN > 0 ? NIN : 1];
#pragma unroll
        for (int i = 0; i < NIN; ++i) vin[i] = reinterpret_cast<const T2*>(a.in[i])[g];
        T in0[NIN > 0 ? NIN : 1], in1[NIN > 0 ? NIN : 1];
#pragma unroll
        for (int i = 0; i < NIN; ++i) {
            in0[i] = vin[i].x;
            in1[i] = vin[i].y;
        }
        T o0[NOUT > 0 ? NOUT : 1], o1[NOUT > 0 ? NOUT : 1];
        f(in0, o0, acc);
        f(in1, o1, acc);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) reinterpret_cast<T2*>(a.out[o])[g] = mk(o0[o], o1[o]);
    }
    // an odd last point
    if ((a.npts & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long g = a.npts - 1;
        T vin[NIN > 0 ? NIN : 1];
#pragma unroll
        for (int i = 0; i < NIN; ++i) vin[i] = a.in[i][g];
        T vout[NOUT > 0 ? NOUT : 1];
        f(vin, vout, acc);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) a.out[o][g] = vout[o];
    }
    if constexpr (NR > 0) block_reduce_store<NR>(acc, a.partials, blockIdx.x);
}

// ----------------------------------------------------------------------------
// x stage, inverse: half spectrum (kx < nx_in, zero above) -> real line.
// ----------------------------------------------------------------------------
template <typename T>
struct XInvArgs {
    int n, nx_in, lx;
    const cpx<T>* in[MAX_ARR];
    T* out[MAX_ARR];
    FftPlan plan_half;
    int tw_n_off;
    const cpx<double>* tw;
    long nlines = 0;  // lines processed (planes * n for a slab)
    int px = 0;       // row pitch of the inputs in elements (0: nx_in); compile-time kernels only
};

template <typename T>
__global__ void __launch_bounds__(256) xinv_kernel(XInvArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, h = n / 2, lx = a.lx;
    const int arr = blockIdx.y;
    cpx<T>* X = reinterpret_cast<cpx<T>*>(smem_raw);  // (h+1) x lx
    cpx<T>* bufA = X + (long)(h + 1) * lx;             // h x lx
    cpx<T>* bufB = bufA + (long)h * lx;
    const long line0 = (long)blockIdx.x * lx;
    const cpx<T>* src = a.in[arr];
    for (int p = threadIdx.x; p < lx * (h + 1); p += blockDim.x) {
        const int l = p / (h + 1), k = p - l * (h + 1);
        cpx<T> v = k < a.nx_in ? src[(line0 + l) * a.nx_in + k] : czero<T>();
        // c2c + REAL() (function_ops.f90, e.g. 3186) keeps the Hermitian part of
        // a spectrum: on the kx = 0 and kx = n/2 columns that is the real part
        if (k == 0 || k == h) v.y = T(0);
        X[(long)k * lx + l] = v;
    }
    __syncthreads();
    const double2* twn = reinterpret_cast<const double2*>(a.tw + a.tw_n_off);
    for (int p = threadIdx.x; p < lx * h; p += blockDim.x) {
        const int k = p / lx, l = p - k * lx;
        const cpx<T> xk = X[(long)k * lx + l];
        const cpx<T> xc = conj(X[(long)(h - k) * lx + l]);
        const cpx<T> Fk = xk + xc;
        const double2 w = __ldg(twn + k);  // exp(-2 pi i k/n); need exp(+...)
        const cpx<T> G = (xk - xc) * mk<T>((T)w.x, (T)(-w.y));
        bufA[(long)k * lx + l] = Fk + mk<T>(-G.y, G.x);  // F + i G
    }
    __syncthreads();
    cpx<T>* z = fft_lines<+1, T>(bufA, bufB, a.plan_half, lx, lx, a.tw, threadIdx.x, blockDim.x);
    T* dst = a.out[arr];
    for (int p = threadIdx.x; p < lx * h; p += blockDim.x) {
        const int l = p / h, m = p - l * h;
        const cpx<T> v = z[(long)m * lx + l];
        reinterpret_cast<cpx<T>*>(dst + (line0 + l) * n)[m] = v;
    }
}

// ----------------------------------------------------------------------------
// Complex x pass (c2c along x, full length) for the fftfwd/fftbwd API.
// ----------------------------------------------------------------------------
template <typename T>
struct XC2CArgs {
    int n, lx;
    const cpx<T>* in;
    cpx<T>* out;
    FftPlan plan;
    const cpx<double>* tw;
    double scale;
};

template <int SIGN, typename T>
__global__ void __launch_bounds__(256) xc2c_kernel(XC2CArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, lx = a.lx;
    cpx<T>* bufA = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* bufB = bufA + (long)n * lx;
    const long line0 = (long)blockIdx.x * lx;
    for (int p = threadIdx.x; p < lx * n; p += blockDim.x) {
        const int l = p / n, x = p - l * n;
        bufA[(long)x * lx + l] = a.in[(line0 + l) * n + x];
    }
    __syncthreads();
    cpx<T>* r = fft_lines<SIGN, T>(bufA, bufB, a.plan, lx, lx, a.tw, threadIdx.x, blockDim.x);
    for (int p = threadIdx.x; p < lx * n; p += blockDim.x) {
        const int l = p / n, x = p - l * n;
        a.out[(line0 + l) * n + x] = r[(long)x * lx + l] * (T)a.scale;
    }
}

// ----------------------------------------------------------------------------
// y pass.  Forward: [z][y<n][kx] -> [z][ky'<nb][kx] (rows outside the band
// dropped).  Inverse: [z][ky'][kx] (zero-padded) -> [z][y<n][kx].
// grid = (ceil(nx/tx), n, narr)
// ----------------------------------------------------------------------------
template <typename T>
struct YArgs {
    int n, nx, tx;       // nx = columns processed (and the row stride of both sides)
    Band band;           // ky band
    const cpx<T>* in[MAX_ARR];
    cpx<T>* out[MAX_ARR];
    FftPlan plan;
    const cpx<double>* tw;
    int nz = 0;          // z planes processed (a slab), n for a whole array
    int px = 0;          // row pitch of both sides in elements (0: nx); compile-time kernels only
};

template <int SIGN, typename T>
__global__ void __launch_bounds__(256) ypass_kernel(YArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb;
    cpx<T>* bufA = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* bufB = bufA + (long)n * tx;
    const int kx0 = blockIdx.x * tx;
    const int z = blockIdx.y;
    const int arr = blockIdx.z;
    const int w = min(tx, nx - kx0);
    const cpx<T>* src = a.in[arr];
    cpx<T>* dst = a.out[arr];
    if (SIGN < 0) {
        for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
            const int y = p / tx, l = p - y * tx;
            bufA[p] = l < w ? src[((long)z * n + y) * nx + kx0 + l] : czero<T>();
        }
    } else {
        for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
            const int fi = p / tx, l = p - fi * tx;
            const int ci = band_compact_index(a.band, fi);
            bufA[p] = (l < w && ci >= 0) ? src[((long)z * nb + ci) * nx + kx0 + l] : czero<T>();
        }
    }
    __syncthreads();
    cpx<T>* r = fft_lines<SIGN, T>(bufA, bufB, a.plan, tx, tx, a.tw, threadIdx.x, blockDim.x);
    if (SIGN < 0) {
        for (int p = threadIdx.x; p < nb * tx; p += blockDim.x) {
            const int ci = p / tx, l = p - ci * tx;
            if (l < w) dst[((long)z * nb + ci) * nx + kx0 + l] = r[(long)band_fft_index(a.band, ci) * tx + l];
        }
    } else {
        for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
            const int y = p / tx, l = p - y * tx;
            if (l < w) dst[((long)z * n + y) * nx + kx0 + l] = r[p];
        }
    }
}

// ----------------------------------------------------------------------------
// Spectral symbols.  K_j = 2 pi j (initialize.f90:170-192).  On a full band the
// Nyquist index of an axis contributes nothing to an odd (first-derivative)
// factor: c2c followed by REAL() keeps only the Hermitian part
// (function_ops.f90:3186 etc.), which cancels it.
// ----------------------------------------------------------------------------
enum Sym : int {
    SYM_ZERO = 0,
    SYM_ONE,
    SYM_IKX,
    SYM_IKY,
    SYM_IKZ,
    SYM_NEG_KSQ,      // laplacian: -|K|^2
    SYM_INV_KSQ,      // +1/|K|^2, 0 at k=0
    SYM_NEG_INV_KSQ,  // -1/|K|^2, 0 at k=0 (solve_poisson with l=1)
    SYM_KK_KSQ,       // + K_a K_b / |K|^2 (a,b from sym_ab), 0 at k=0
};

struct Kvec {
    double kx, ky, kz;        // true wavenumbers
    double ox, oy, oz;        // odd-factor wavenumbers (0 at a Nyquist index)
    double ksq;
};

__device__ __forceinline__ Kvec make_k(int n, int fx, int fy, int fz) {
    const double twopi = 2.0 * 3.14159265358979311600;  // 2.0_pr*PI, PI = 4 atan2(1,1)
    Kvec k;
    const int jx = signed_j(n, fx), jy = signed_j(n, fy), jz = signed_j(n, fz);
    k.kx = twopi * (double)jx;
    k.ky = twopi * (double)jy;
    k.kz = twopi * (double)jz;
    const bool even = (n & 1) == 0;
    k.ox = (even && fx == n / 2) ? 0.0 : k.kx;
    k.oy = (even && fy == n / 2) ? 0.0 : k.ky;
    k.oz = (even && fz == n / 2) ? 0.0 : k.kz;
    k.ksq = k.kx * k.kx + k.ky * k.ky + k.kz * k.kz;
    return k;
}

__device__ __forceinline__ cpx<double> apply_sym(int sym, int ab, const Kvec& k, cpx<double> v) {
    switch (sym) {
        case SYM_ZERO: return mk(0.0, 0.0);
        case SYM_ONE: return v;
        case SYM_IKX: return mk(-k.ox * v.y, k.ox * v.x);
        case SYM_IKY: return mk(-k.oy * v.y, k.oy * v.x);
        case SYM_IKZ: return mk(-k.oz * v.y, k.oz * v.x);
        case SYM_NEG_KSQ: return v * (-k.ksq);
        case SYM_INV_KSQ: return k.ksq == 0.0 ? mk(0.0, 0.0) : v * (1.0 / k.ksq);
        case SYM_NEG_INV_KSQ: return k.ksq == 0.0 ? mk(0.0, 0.0) : v * (-1.0 / k.ksq);
        case SYM_KK_KSQ: {
            if (k.ksq == 0.0) return mk(0.0, 0.0);
            const int ia = ab / 3, ib = ab % 3;
            const double ka = ia == 0 ? k.ox : (ia == 1 ? k.oy : k.oz);
            const double kb = ib == 0 ? k.ox : (ib == 1 ? k.oy : k.oz);
            return v * (ka * kb / k.ksq);
        }
    }
    return v;
}

__device__ __forceinline__ cpx<double> ld_spec(const void* p, int f64, long idx) {
    if (f64) {
        const double2 v = reinterpret_cast<const double2*>(p)[idx];
        return mk(v.x, v.y);
    }
    const float2 v = reinterpret_cast<const float2*>(p)[idx];
    return mk((double)v.x, (double)v.y);
}
__device__ __forceinline__ void st_spec(void* p, int f64, long idx, cpx<double> v) {
    if (f64)
        reinterpret_cast<double2*>(p)[idx] = make_double2(v.x, v.y);
    else
        reinterpret_cast<float2*>(p)[idx] = make_float2((float)v.x, (float)v.y);
}
// Parseval weight of a half-spectrum column (real fields)
__device__ __forceinline__ double kx_weight(int n, int fx) { return (fx == 0 || 2 * fx == n) ? 1.0 : 2.0; }

// State-vector storage: double2 (FP64 path) or float2 (mixed path); the
// spectral state kernels load into double, compute in double and round on
// the store.
template <typename V>
__device__ __forceinline__ double2 ldv(const V* p, long i) {
    const V v = p[i];
    return make_double2((double)v.x, (double)v.y);
}
template <typename V>
__device__ __forceinline__ void stv(V* p, long i, double2 v) {
    p[i] = V{(decltype(p[i].x))v.x, (decltype(p[i].y))v.y};
}
// v as the storage V rounds it (what ldv returns after stv)
template <typename V>
__device__ __forceinline__ double2 rndv(double2 v) {
    const V r{(decltype(V{}.x))v.x, (decltype(V{}.y))v.y};
    return make_double2((double)r.x, (double)r.y);
}

// ----------------------------------------------------------------------------
// z stage, forward (optionally round trip).  grid = (ceil(nx/tx), nb, narr).
// For each array: z FFT, keep |kz| <= cut, scale 1/N^3, multiply by `sym`,
// add coef*add_sym*add_spec, reductions, write the pruned spectrum and/or
// transform back along z into ys_out.
// ----------------------------------------------------------------------------
struct ZFwdOp {
    const void* in;       // ys array, work type
    void* spec_out;       // optional pruned spectrum
    int spec_f64;
    void* ys_out;         // optional round-trip output (work type)
    int sym, sym_ab;
    const void* add;      // optional second term
    int add_f64, add_sym, add_ab;
    double add_coef;
    int red_self;               // slot for sum w|Y|^2, -1 none
    const void* red_with[3];    // sum w Re(Y conj(W_i)) into red_with_slot[i] (null: none)
    int red_with_f64[3], red_with_slot[3];
};

template <typename T>
struct ZFwdArgs {
    int n, nx, tx;
    Band band;
    ZFwdOp op[MAX_ARR];
    FftPlan plan;
    const cpx<double>* tw;
    double* partials;  // [blocks][MAX_RED]
    double norm;       // 1/N^3
    int px = 0;        // row pitch of the y-stage arrays (0: nx); spectra keep pitch nx
};

template <typename T>
__global__ void __launch_bounds__(256) zfwd_kernel(ZFwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb;
    cpx<T>* bufA = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* bufB = bufA + (long)n * tx;
    const int kx0 = blockIdx.x * tx;
    const int cy = blockIdx.y;
    const ZFwdOp& op = a.op[blockIdx.z];
    const int w = min(tx, nx - kx0);
    const cpx<T>* src = reinterpret_cast<const cpx<T>*>(op.in);
    const long plane = (long)nb * nx;
    for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
        const int z = p / tx, l = p - z * tx;
        bufA[p] = l < w ? src[(long)z * plane + (long)cy * nx + kx0 + l] : czero<T>();
    }
    __syncthreads();
    cpx<T>* r = fft_lines<-1, T>(bufA, bufB, a.plan, tx, tx, a.tw, threadIdx.x, blockDim.x);
    cpx<T>* o = (r == bufA) ? bufB : bufA;  // free buffer for the round trip
    double acc[MAX_RED];
#pragma unroll
    for (int i = 0; i < MAX_RED; ++i) acc[i] = 0.0;
    const int fy = band_fft_index(a.band, cy);
    for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
        const int fz = p / tx, l = p - fz * tx;
        const int cz = band_compact_index(a.band, fz);
        cpx<double> Y = mk(0.0, 0.0);
        if (cz >= 0 && l < w) {
            const int fx = kx0 + l;
            const Kvec k = make_k(n, fx, fy, fz);
            const cpx<T> v = r[p];
            Y = apply_sym(op.sym, op.sym_ab, k, mk((double)v.x, (double)v.y) * a.norm);
            const long si = ((long)cz * nb + cy) * nx + fx;
            if (op.add) Y = Y + apply_sym(op.add_sym, op.add_ab, k, ld_spec(op.add, op.add_f64, si)) * op.add_coef;
            const double wgt = kx_weight(n, fx);
            if (op.red_self >= 0) acc[op.red_self] += wgt * (Y.x * Y.x + Y.y * Y.y);
            for (int r = 0; r < 3; ++r)
                if (op.red_with[r]) {
                    const cpx<double> W = ld_spec(op.red_with[r], op.red_with_f64[r], si);
                    acc[op.red_with_slot[r]] += wgt * (Y.x * W.x + Y.y * W.y);
                }
            if (op.spec_out) st_spec(op.spec_out, op.spec_f64, si, Y);
        }
        if (op.ys_out) o[p] = mk((T)Y.x, (T)Y.y);
    }
    const int block_lin = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    block_reduce_store<MAX_RED>(acc, a.partials, block_lin);
    if (op.ys_out) {
        __syncthreads();
        cpx<T>* other = (o == bufA) ? bufB : bufA;
        cpx<T>* q = fft_lines<+1, T>(o, other, a.plan, tx, tx, a.tw, threadIdx.x, blockDim.x);
        cpx<T>* dst = reinterpret_cast<cpx<T>*>(op.ys_out);
        for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
            const int z = p / tx, l = p - z * tx;
            if (l < w) dst[(long)z * plane + (long)cy * nx + kx0 + l] = q[p];
        }
    }
}

// ----------------------------------------------------------------------------
// z stage, inverse from spectra: out = IFFT_z( sum_s coef_s * sym_s(k) spec_s ).
// grid = (ceil(nx/tx), nb, narr)
// ----------------------------------------------------------------------------
struct ZSrc {
    const void* spec;
    int f64, sym, ab;
    double coef;
};
struct ZInvOp {
    ZSrc src[3];
    int nsrc;
    void* ys_out;
};

template <typename T>
struct ZInvArgs {
    int n, nx, tx;
    Band band;
    ZInvOp op[MAX_ARR];
    FftPlan plan;
    const cpx<double>* tw;
    int px = 0;  // row pitch of the y-stage arrays (0: nx); spectra keep pitch nx
};

// One spectrum, up to four symbols: the z inverse of a field and of its
// derivatives (u and grad u, p and grad p, ...) from one load of the source
constexpr int ZMULTI = 4;
struct ZInvMultiOp {
    const void* spec;
    int f64, nout;
    int sym[ZMULTI], ab[ZMULTI];
    double coef[ZMULTI];
    void* ys_out[ZMULTI];
};
template <typename T>
struct ZInvMultiArgs {
    int n, nx;
    Band band;
    ZInvMultiOp op[MAX_ARR];
    int px = 0;  // row pitch of the y-stage arrays (0: nx); spectra keep pitch nx
};

template <typename T>
__global__ void __launch_bounds__(256) zinv_kernel(ZInvArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb;
    cpx<T>* bufA = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* bufB = bufA + (long)n * tx;
    const int kx0 = blockIdx.x * tx;
    const int cy = blockIdx.y;
    const ZInvOp& op = a.op[blockIdx.z];
    const int w = min(tx, nx - kx0);
    const int fy = band_fft_index(a.band, cy);
    for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
        const int fz = p / tx, l = p - fz * tx;
        const int cz = band_compact_index(a.band, fz);
        cpx<double> Y = mk(0.0, 0.0);
        if (cz >= 0 && l < w) {
            const int fx = kx0 + l;
            const Kvec k = make_k(n, fx, fy, fz);
            const long si = ((long)cz * nb + cy) * nx + fx;
            for (int s = 0; s < op.nsrc; ++s)
                Y = Y + apply_sym(op.src[s].sym, op.src[s].ab, k, ld_spec(op.src[s].spec, op.src[s].f64, si)) *
                            op.src[s].coef;
        }
        bufA[p] = mk((T)Y.x, (T)Y.y);
    }
    __syncthreads();
    cpx<T>* q = fft_lines<+1, T>(bufA, bufB, a.plan, tx, tx, a.tw, threadIdx.x, blockDim.x);
    cpx<T>* dst = reinterpret_cast<cpx<T>*>(op.ys_out);
    const long plane = (long)nb * nx;
    for (int p = threadIdx.x; p < n * tx; p += blockDim.x) {
        const int z = p / tx, l = p - z * tx;
        if (l < w) dst[(long)z * plane + (long)cy * nx + kx0 + l] = q[p];
    }
}

// ----------------------------------------------------------------------------
// Spectral-state kernels on pruned FP64 vector spectra [3][nb][nb][nx].
// ----------------------------------------------------------------------------
struct SpecGeom {
    int n, nx, nb;
    Band band;
    long ncomp;  // nb*nb*nx
};

__device__ __forceinline__ void spec_coords(const SpecGeom& g, long i, int& fx, int& fy, int& fz) {
    const int cx = (int)(i % g.nx);
    const long t = i / g.nx;
    const int cy = (int)(t % g.nb);
    const int cz = (int)(t / g.nb);
    fx = cx;
    fy = band_fft_index(g.band, cy);
    fz = band_fft_index(g.band, cz);
}

// out = a*x + b*y + c*z  (any pointer may alias out; y/z may be null)
template <typename V>
__global__ void spec_lincomb_kernel(SpecGeom g, V* out, double a, const V* x, double b, const V* y, double c,
                                    const V* z) {
    const long nt = 3 * g.ncomp;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += (long)gridDim.x * blockDim.x) {
        double2 v = ldv(x, i);
        double2 r = make_double2(a * v.x, a * v.y);
        if (y) {
            const double2 w = ldv(y, i);
            r.x += b * w.x;
            r.y += b * w.y;
        }
        if (z) {
            const double2 w = ldv(z, i);
            r.x += c * w.x;
            r.y += c * w.y;
        }
        stv(out, i, r);
    }
}

// out = coef[0]^pw * in over n elements of type C (complex float / double),
// the factor read from device memory (stays valid in a replayed graph)
template <typename C>
__global__ void spec_scale_pow_kernel(C* out, const C* in, long n, const double* coef, int pw) {
    double f = 1.0;
    for (int k = 0; k < pw; ++k) f *= coef[0];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const C v = in[i];
        out[i] = C{(decltype(v.x))(f * v.x), (decltype(v.y))(f * v.y)};
    }
}

// out = c0 a + c1 b + c2 c over n elements of type C (a polynomial in tau of
// three coefficient spectra); with coef non-null the coefficients are
// cs^2 (1, tau, tau^2) for cs = coef[0], tau = coef[1], read from device
// memory (stays valid in a replayed graph)
template <typename C>
__global__ void spec_poly3_kernel(C* out, const C* a, const C* b, const C* c, long n, double c0, double c1,
                                  double c2, const double* coef) {
    if (coef) {
        c0 = coef[0] * coef[0];
        c1 = c0 * coef[1];
        c2 = c1 * coef[1];
    }
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const C x = a[i], y = b[i], z = c[i];
        out[i] = C{(decltype(x.x))(c0 * x.x + c1 * y.x + c2 * z.x), (decltype(x.y))(c0 * x.y + c1 * y.y + c2 * z.y)};
    }
}

// The vector transport's two outputs and the retraction in one pass over the
// state (function_ops.f90:1716-1768 with optimization.f90:324-338):
//   tg = ag g + bg u + cg d,  td = ad d + bd u + cd d,  u <- cs u + ct d
template <typename V>
__global__ void spec_transport_kernel(long nt, const V* g, const V* d, V* u, V* tg, V* td, double ag, double bg,
                                      double cg, double ad, double bd, double cd, double cs, double ct) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += (long)gridDim.x * blockDim.x) {
        const double2 gv = ldv(g, i), dv = ldv(d, i), uv = ldv(u, i);
        stv(tg, i, make_double2(ag * gv.x + bg * uv.x + cg * dv.x, ag * gv.y + bg * uv.y + cg * dv.y));
        stv(td, i, make_double2(ad * dv.x + bd * uv.x + cd * dv.x, ad * dv.y + bd * uv.y + cd * dv.y));
        stv(u, i, make_double2(cs * uv.x + ct * dv.x, cs * uv.y + ct * dv.y));
    }
}

// Row-structured walk over a band spectrum [nb][nb][nx]: block b takes rows
// r = b, b + gridDim.x, ... (r = cz*nb + cy), threads take kx; no division per
// element.  Signed indices and |j|^2 of a mode give the wavenumbers exactly
// as make_k does (K = 2 pi j).
struct SpecRow {
    int cz, cy, jy, jz;
    __device__ __forceinline__ SpecRow(const SpecGeom& g, int r) {
        cz = r / g.nb;
        cy = r - cz * g.nb;
        jy = signed_j(g.n, band_fft_index(g.band, cy));
        jz = signed_j(g.n, band_fft_index(g.band, cz));
    }
};

// f <- Leray(s(K) * scale * f) over a band spectrum, either part optional:
// the Hilbert gradient symbol s = 1/(1+(lambda1|K|)^(2 order))
// (function_ops.f90:3611) read from a table indexed by |j|^2, and divAvg_free
// (2843-2918): u - K(K.u)/|K|^2 (odd factors), k = 0 -> 0.
// f <- Leray(s f) at one mode (ox, oy, oz: the odd-factor wavenumbers, 0 at a
// Nyquist index; ksq = |K|^2), the mode k = 0 set to 0
__device__ __forceinline__ void hilbert_leray_point(double2& u0, double2& u1, double2& u2, double s, bool leray,
                                                    double ox, double oy, double oz, double ksq) {
    u0.x *= s; u0.y *= s;
    u1.x *= s; u1.y *= s;
    u2.x *= s; u2.y *= s;
    if (leray) {
        if (ksq > MACH_EPSILON) {
            const double dr = ox * u0.x + oy * u1.x + oz * u2.x;
            const double di = ox * u0.y + oy * u1.y + oz * u2.y;
            const double is = 1.0 / ksq;
            u0.x -= ox * dr * is; u0.y -= ox * di * is;
            u1.x -= oy * dr * is; u1.y -= oy * di * is;
            u2.x -= oz * dr * is; u2.y -= oz * di * is;
        } else {
            u0 = u1 = u2 = make_double2(0.0, 0.0);
        }
    }
}

template <typename V>
__global__ void spec_hilbert_leray_kernel(SpecGeom g, V* f, const double* __restrict__ htab, double scale,
                                          int do_leray) {
    const double twopi = 2.0 * 3.14159265358979311600;
    const int nrows = g.nb * g.nb;
    // one warp per row (kx across the lanes), blockDim / 32 rows per block pass
    const int lane = threadIdx.x & 31, rows_per = blockDim.x >> 5;
    for (int r = blockIdx.x * rows_per + (threadIdx.x >> 5); r < nrows; r += gridDim.x * rows_per) {
        const SpecRow row(g, r);
        const long base = (long)r * g.nx;
        const double ky = twopi * (double)row.jy, kz = twopi * (double)row.jz;
        const double oy = (2 * band_fft_index(g.band, row.cy) == g.n) ? 0.0 : ky;
        const double oz = (2 * band_fft_index(g.band, row.cz) == g.n) ? 0.0 : kz;
        for (int fx = lane; fx < g.nx; fx += 32) {
            const long i = base + fx;
            double2 u0 = ldv(f, i), u1 = ldv(f, g.ncomp + i), u2 = ldv(f, 2 * g.ncomp + i);
            double s = scale;
            if (htab) s *= htab[fx * fx + row.jy * row.jy + row.jz * row.jz];
            const double kx = twopi * (double)fx;
            const double ox = (2 * fx == g.n) ? 0.0 : kx;
            hilbert_leray_point(u0, u1, u2, s, do_leray != 0, ox, oy, oz, kx * kx + ky * ky + kz * kz);
            stv(f, i, u0);
            stv(f, g.ncomp + i, u1);
            stv(f, 2 * g.ncomp + i, u2);
        }
    }
}

// Hilbert gradient + Leray projection of two fields (f1 scaled by s1, f2 by
// s2) and, on the results, the H inner products <f2, f1> and <f2, f2> (the
// weights of spec_dot_kernel's kind 1) as per-block partials [block][2]
template <typename V>
__global__ void __launch_bounds__(128) spec_hilbert_leray_pair_dot_kernel(SpecGeom g, V* f1, double s1, V* f2,
                                                                       double s2, const double* __restrict__ htab,
                                                                       const double* __restrict__ hwtab,
                                                                       double* partials) {
    const double twopi = 2.0 * 3.14159265358979311600;
    const int nrows = g.nb * g.nb;
    double acc[2] = {0.0, 0.0};
    // one warp per row (kx across the lanes), blockDim / 32 rows per block pass
    const int lane = threadIdx.x & 31, rows_per = blockDim.x >> 5;
    for (int r = blockIdx.x * rows_per + (threadIdx.x >> 5); r < nrows; r += gridDim.x * rows_per) {
        const SpecRow row(g, r);
        const long base = (long)r * g.nx;
        const double ky = twopi * (double)row.jy, kz = twopi * (double)row.jz;
        const double oy = (2 * band_fft_index(g.band, row.cy) == g.n) ? 0.0 : ky;
        const double oz = (2 * band_fft_index(g.band, row.cz) == g.n) ? 0.0 : kz;
        const int jyz = row.jy * row.jy + row.jz * row.jz;
        for (int fx = lane; fx < g.nx; fx += 32) {
            const long i = base + fx;
            double2 a0 = ldv(f1, i), a1 = ldv(f1, g.ncomp + i), a2 = ldv(f1, 2 * g.ncomp + i);
            double2 b0 = ldv(f2, i), b1 = ldv(f2, g.ncomp + i), b2 = ldv(f2, 2 * g.ncomp + i);
            const double h = htab[fx * fx + jyz];
            const double kx = twopi * (double)fx;
            const double ox = (2 * fx == g.n) ? 0.0 : kx;
            const double ksq = kx * kx + ky * ky + kz * kz;
            hilbert_leray_point(a0, a1, a2, s1 * h, true, ox, oy, oz, ksq);
            hilbert_leray_point(b0, b1, b2, s2 * h, true, ox, oy, oz, ksq);
            stv(f1, i, a0);
            stv(f1, g.ncomp + i, a1);
            stv(f1, 2 * g.ncomp + i, a2);
            stv(f2, i, b0);
            stv(f2, g.ncomp + i, b1);
            stv(f2, 2 * g.ncomp + i, b2);
            const double w = kx_weight(g.n, fx) * hwtab[fx * fx + jyz];
            acc[0] += w * ((b0.x * a0.x + b0.y * a0.y) + (b1.x * a1.x + b1.y * a1.y) + (b2.x * a2.x + b2.y * a2.y));
            acc[1] += w * ((b0.x * b0.x + b0.y * b0.y) + (b1.x * b1.x + b1.y * b1.y) + (b2.x * b2.x + b2.y * b2.y));
        }
    }
    block_reduce_store<2>(acc, partials, blockIdx.x);
}

// The search direction from the projected gradient: g <- sg g, then
// d <- g + beta td (td may be null: d <- g)
template <typename V>
__global__ void spec_direction_kernel(long nt, V* g, double sg, V* d, double beta, const V* td) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += (long)gridDim.x * blockDim.x) {
        double2 v = ldv(g, i);
        v.x *= sg;
        v.y *= sg;
        stv(g, i, v);
        if (td) {
            const double2 w = ldv(td, i);
            v.x += beta * w.x;
            v.y += beta * w.y;
        }
        stv(d, i, v);
    }
}

// Up to 8 vector inner products in one pass.  kind: 0 L2, 1 H_l weight
// (1+(lambda1|K|)^order)^2 (function_ops.f90:3472), 2 divergence energy
// |K_odd . f|^2, 3 curl energy |K x f|^2, 4 |K|^4 |f|^2 (kinds 2-4 read
// pair.a only).
struct SpecDotPair {
    const void* a;  // state vectors (double2 or float2 storage, the kernel's V)
    const void* b;
    int kind;
};
struct SpecDotArgs {
    SpecGeom g;
    SpecDotPair pr[8];
    int npairs;
    // optional ax_out <- ax_x + ax_a ax_y before the products (the pairs may
    // read ax_out: each element is updated by the thread that then reads it)
    void* ax_out = nullptr;
    const void* ax_x = nullptr;
    const void* ax_y = nullptr;
    double ax_a = 0.0;
    // the distinct vectors of the pass for spec_dot_fixed_kernel, ax_out
    // last when the pass reads it (ax_last)
    const void* vec[8];
    int ax_last = 0;
    const double* hwtab;  // H_l weight (1+(lambda1|K|)^order)^2 by |j|^2 (function_ops.f90:3472), or null
    double* partials;
};

// One product of a pair at a mode (u = pair.a, w = pair.b there; K = 2 pi
// (ox, oy, oz) / 2 pi with the Nyquist components zeroed).
__device__ __forceinline__ double dot_term(int kind, const double2 (&u)[3], const double2 (&w)[3], double ox,
                                           double oy, double oz, double hw) {
    if (kind == 3) {
        // |K x a|^2 (vel2vort, function_ops.f90:2485-2495); in-band modes
        // have no Nyquist index, so K = 2 pi j on every axis
        const double w0r = oy * u[2].x - oz * u[1].x, w0i = oy * u[2].y - oz * u[1].y;
        const double w1r = oz * u[0].x - ox * u[2].x, w1i = oz * u[0].y - ox * u[2].y;
        const double w2r = ox * u[1].x - oy * u[0].x, w2i = ox * u[1].y - oy * u[0].y;
        return w0r * w0r + w0i * w0i + w1r * w1r + w1i * w1i + w2r * w2r + w2i * w2i;
    }
    if (kind == 4) {  // |K|^4 |a|^2 (||Lap a||^2)
        const double k2 = ox * ox + oy * oy + oz * oz;
        double m2 = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) m2 += u[c].x * u[c].x + u[c].y * u[c].y;
        return k2 * k2 * m2;
    }
    if (kind == 2) {  // |K_odd . a|^2
        const double dr = ox * u[0].x + oy * u[1].x + oz * u[2].x;
        const double di = ox * u[0].y + oy * u[1].y + oz * u[2].y;
        return dr * dr + di * di;
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) s += u[c].x * w[c].x + u[c].y * w[c].y;
    return kind == 1 ? hw * s : s;
}

// Up to 8 inner products with every pair's vectors loaded per pair (any
// pattern of operands).  One warp per row, each lane one mode at a time.
template <typename V>
__global__ void __launch_bounds__(RED_THREADS) spec_dot_kernel(SpecDotArgs a) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const SpecGeom& g = a.g;
    const double twopi = 2.0 * 3.14159265358979311600;
    const int nrows = g.nb * g.nb;
    const int lane = threadIdx.x & 31, wrow = threadIdx.x >> 5, rows_per = blockDim.x >> 5;
    for (int r = blockIdx.x * rows_per + wrow; r < nrows; r += gridDim.x * rows_per) {
        const SpecRow row(g, r);
        const long base = (long)r * g.nx;
        const double oy = (2 * band_fft_index(g.band, row.cy) == g.n) ? 0.0 : twopi * (double)row.jy;
        const double oz = (2 * band_fft_index(g.band, row.cz) == g.n) ? 0.0 : twopi * (double)row.jz;
        const int jyz = row.jy * row.jy + row.jz * row.jz;
        for (int fx = lane; fx < g.nx; fx += 32) {
            const long i = base + fx;
            const double wgt = kx_weight(g.n, fx);
            const double hw = a.hwtab ? a.hwtab[fx * fx + jyz] : 1.0;
            const double ox = (2 * fx == g.n) ? 0.0 : twopi * (double)fx;
            if (a.ax_out) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const long k = c * g.ncomp + i;
                    const double2 x = ldv((const V*)a.ax_x, k), y = ldv((const V*)a.ax_y, k);
                    stv((V*)a.ax_out, k, make_double2(x.x + a.ax_a * y.x, x.y + a.ax_a * y.y));
                }
            }
            // unrolled to the bound of 8 so that acc stays in registers
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                if (p >= a.npairs) break;
                const SpecDotPair& q = a.pr[p];
                double2 u[3], w[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) u[c] = ldv((const V*)q.a, c * g.ncomp + i);
#pragma unroll
                for (int c = 0; c < 3; ++c) w[c] = q.kind < 2 ? ldv((const V*)q.b, c * g.ncomp + i) : u[c];
                acc[p] += wgt * dot_term(q.kind, u, w, ox, oy, oz, hw);
            }
        }
    }
    block_reduce_store<8>(acc, a.partials, blockIdx.x);
}

// The same products for a pattern of operands fixed at compile time: the NV
// distinct vectors are loaded once per mode, pair p reads vec[(PAT >> 6p) & 7]
// and vec[(PAT >> (6p + 3)) & 7], and the optional update reads
// vec[(PAT >> 48) & 7] + ax_a vec[(PAT >> 51) & 7] and writes ax_out (which
// replaces vec[NV - 1] when ax_last).
template <typename V, int NV, int NP, unsigned long long PAT>
__global__ void __launch_bounds__(RED_THREADS) spec_dot_fixed_kernel(SpecDotArgs a) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const SpecGeom& g = a.g;
    const double twopi = 2.0 * 3.14159265358979311600;
    const int nrows = g.nb * g.nb;
    constexpr int XI = (int)((PAT >> 48) & 7), YI = (int)((PAT >> 51) & 7);
    // ax_out is read before it is written only when it is an operand of the update
    const bool load_last = !(a.ax_out && a.ax_last && XI != NV - 1 && YI != NV - 1);
    const int lane = threadIdx.x & 31, wrow = threadIdx.x >> 5, rows_per = blockDim.x >> 5;
    for (int r = blockIdx.x * rows_per + wrow; r < nrows; r += gridDim.x * rows_per) {
        const SpecRow row(g, r);
        const long base = (long)r * g.nx;
        const double oy = (2 * band_fft_index(g.band, row.cy) == g.n) ? 0.0 : twopi * (double)row.jy;
        const double oz = (2 * band_fft_index(g.band, row.cz) == g.n) ? 0.0 : twopi * (double)row.jz;
        const int jyz = row.jy * row.jy + row.jz * row.jz;
        for (int fx = lane; fx < g.nx; fx += 32) {
            const long i = base + fx;
            const double wgt = kx_weight(g.n, fx);
            const double hw = a.hwtab ? a.hwtab[fx * fx + jyz] : 1.0;
            const double ox = (2 * fx == g.n) ? 0.0 : twopi * (double)fx;
            double2 x[NV][3];
#pragma unroll
            for (int v = 0; v < NV; ++v)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    x[v][c] = (v < NV - 1 || load_last) ? ldv((const V*)a.vec[v], c * g.ncomp + i)
                                                         : make_double2(0.0, 0.0);
            if (a.ax_out) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double2 nv =
                        rndv<V>(make_double2(x[XI][c].x + a.ax_a * x[YI][c].x, x[XI][c].y + a.ax_a * x[YI][c].y));
                    stv((V*)a.ax_out, c * g.ncomp + i, nv);
                    if (a.ax_last) x[NV - 1][c] = nv;
                }
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const int ia = (int)((PAT >> (6 * p)) & 7), ib = (int)((PAT >> (6 * p + 3)) & 7);
                acc[p] += wgt * dot_term(a.pr[p].kind, x[ia], x[ib], ox, oy, oz, hw);
            }
        }
    }
    block_reduce_store<8>(acc, a.partials, blockIdx.x);
}

// Fourier coefficients of a physical scalar restricted to a band, full-band
// energy outside the band: used to check that a loaded field is band-limited.
// (Implemented with the forward pipeline plus a reduction; see engine.)

}  // namespace mlq
