// cfft.cuh -- FFT pass kernels specialised at compile time for one grid size N.
//
// Every line length, radix sequence, register layout and shared-memory map is
// a compile-time constant, so the only run-time index arithmetic left is the
// work-item decomposition.  A line of length L is held by TPL = L/E threads,
// thread t owning positions t + TPL*m (m < E) in registers before and after
// every stage (Stockham autosort, see regfft.cuh for the generic form).
//
//  * x passes (rows of the physical field): TPL <= 32, so a line lives in one
//    warp and the exchanges between stages need only __syncwarp.  The
//    run-time twiddles of each stage depend only on t and are loaded once per
//    thread into registers; the real-to-half-complex pre/post twiddle
//    W_N^(t + TPL m) = W_N^t * W_N^(TPL m) uses a compile-time constant for
//    the second factor.
//  * y/z passes (columns): lanes walk the contiguous kx axis (TX columns per
//    tile, 128-byte rows), the threads of a column span warps, and exchanges
//    are block-wide.  Twiddles come from a per-block shared-memory table; the
//    lanes of a row share t, so those reads are broadcasts.
//
// All kernels are persistent: a grid of a few blocks per SM walks the work
// items with a fixed stride, so reduction partials are few and their order
// is fixed (deterministic).
#pragma once

#include <type_traits>

#include "functors.cuh"
#include "kernels.cuh"

namespace mlq {

// ----------------------------------------------------------------------------
// Compile-time helpers
// ----------------------------------------------------------------------------
__host__ __device__ constexpr int clog2(int v) {
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}

// sin x and cos x for |x| <= pi/4 by their Taylor series (compile time only;
// the truncation error of 14 terms is below 1e-25).
__host__ __device__ constexpr double ce_sin_small(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double ce_cos_small(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
struct CeCS {
    double c, s;
};
// cos and sin of 2 pi j / M: exact quadrant and octant reduction in integers,
// then the series on an angle of at most pi/4.
__host__ __device__ constexpr CeCS ce_cs2pi(long j, long M) {
    j %= M;
    if (j < 0) j += M;
    const long q = (4 * j) / M;   // quadrant
    const long r = 4 * j - q * M;  // angle within the quadrant = (pi/2) r / M
    const double half_pi = 1.57079632679489661923;
    double cq = 0.0, sq = 0.0;
    if (2 * r <= M) {
        const double x = half_pi * ((double)r / (double)M);
        cq = ce_cos_small(x);
        sq = ce_sin_small(x);
    } else {
        const double x = half_pi * ((double)(M - r) / (double)M);
        cq = ce_sin_small(x);
        sq = ce_cos_small(x);
    }
    if (q == 0) return {cq, sq};
    if (q == 1) return {-sq, cq};
    if (q == 2) return {-cq, -sq};
    return {sq, -cq};
}
// W_M^J = exp(-2 pi i J / M) as a compile-time constant in precision T
template <typename T, long M, long J>
__device__ __forceinline__ cpx<T> cw() {
    constexpr CeCS v = ce_cs2pi(J, M);
    return mk<T>((T)v.c, (T)(-v.s));
}

// compile-time loop: f(std::integral_constant<int, I>) for I in [B, E)
template <int B, int E>
struct SFor {
    template <class F>
    __device__ __forceinline__ static void run(F&& f) {
        if constexpr (B < E) {
            f(std::integral_constant<int, B>{});
            SFor<B + 1, E>::run(f);
        }
    }
};

// a * w (SIGN < 0) or a * conj(w) (SIGN > 0)
template <int SIGN, typename T>
__device__ __forceinline__ cpx<T> cmul_s(cpx<T> a, cpx<T> w) {
    if constexpr (SIGN < 0)
        return mk(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
    else
        return mk(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// ----------------------------------------------------------------------------
// Plan of a length-L transform held as E elements per thread: radix-E stages,
// then one smaller power-of-two radix for the remainder.
// ----------------------------------------------------------------------------
template <int L, int E>
struct CPlan {
    static_assert((L & (L - 1)) == 0 && (E & (E - 1)) == 0 && E >= 2 && E <= 16 && E <= L, "plan shape");
    static constexpr int TPL = L / E;
    static constexpr int LGL = clog2(L), LGE = clog2(E);
    static constexpr int NFULL = LGL / LGE, REMLG = LGL % LGE;
    static constexpr int NST = NFULL + (REMLG ? 1 : 0);
    __host__ __device__ static constexpr int radix(int s) { return s < NFULL ? E : (1 << REMLG); }
    __host__ __device__ static constexpr int ns(int s) {
        int v = 1;
        for (int i = 0; i < s; ++i) v *= radix(i);
        return v;
    }
    // butterflies of stage s whose twiddles differ (1 when ns(s) divides TPL)
    __host__ __device__ static constexpr int qd(int s) { return ns(s) <= TPL ? 1 : E / radix(s); }
    __host__ __device__ static constexpr int twc(int s) { return s == 0 ? 0 : qd(s) * (radix(s) - 1); }
    __host__ __device__ static constexpr int twoff(int s) {
        int o = 0;
        for (int i = 0; i < s; ++i) o += twc(i);
        return o;
    }
    static constexpr int NTW = twoff(NST);
};

// Twiddles of one thread in registers; tab[j] = W_L^j in precision T.
template <int L, int E, typename T>
struct TwReg {
    using P = CPlan<L, E>;
    cpx<T> w[P::NTW > 0 ? P::NTW : 1];
    __device__ __forceinline__ void load(const cpx<T>* __restrict__ tab, int t) {
        SFor<1, P::NST>::run([&](auto sc) {
            constexpr int S = decltype(sc)::value;
            constexpr int R = P::radix(S), NS = P::ns(S), QD = P::qd(S), STEP = L / (NS * R);
            SFor<0, QD>::run([&](auto ic) {
                constexpr int I = decltype(ic)::value;
                const int k = (t + P::TPL * I) & (NS - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) w[P::twoff(S) + I * (R - 1) + r - 1] = tab[r * k * STEP];
            });
        });
    }
    template <int S, int I, int RI>
    __device__ __forceinline__ cpx<T> get(int) const {
        constexpr int QD = P::qd(S), R = P::radix(S);
        return w[P::twoff(S) + (QD == 1 ? 0 : I) * (R - 1) + RI - 1];
    }
};

// Twiddles read from a table W_L^j (shared memory) at run time.
template <int L, int E, typename T>
struct TwTab {
    using P = CPlan<L, E>;
    const cpx<T>* tab;
    template <int S, int I, int RI>
    __device__ __forceinline__ cpx<T> get(int k) const {
        constexpr int R = P::radix(S), NS = P::ns(S), STEP = L / (NS * R);
        return tab[RI * k * STEP];
    }
};

// Stage-major twiddles in shared memory: stage S holds W_L^(r k STEP) at
// off(S) + (r - 1) NS + k, so threads with consecutive k (the threads of one
// exchange row) read consecutive words, free of bank conflicts (a table
// indexed r k STEP strides by STEP words).  At most L entries.
template <int L, int E, typename T>
struct TwStage {
    using P = CPlan<L, E>;
    __host__ __device__ static constexpr int off(int s) {
        int o = 0;
        for (int i = 1; i < s; ++i) o += (P::radix(i) - 1) * P::ns(i);
        return o;
    }
    static constexpr int SIZE = off(P::NST);
    static_assert(SIZE <= L, "stage tables fit in L entries");
    const cpx<T>* tab;
    // fill from the table W_L^j (global memory); every thread of the block calls it
    __device__ __forceinline__ static void fill(cpx<T>* dst, const cpx<T>* __restrict__ twL) {
        SFor<1, P::NST>::run([&](auto sc) {
            constexpr int S = decltype(sc)::value;
            constexpr int R = P::radix(S), NS = P::ns(S), STEP = L / (NS * R);
            for (int j = threadIdx.x; j < (R - 1) * NS; j += blockDim.x) {
                const int r = j / NS + 1, k = j - (r - 1) * NS;
                dst[off(S) + j] = twL[r * k * STEP];
            }
        });
    }
    template <int S, int I, int RI>
    __device__ __forceinline__ cpx<T> get(int k) const {
        return tab[off(S) + (RI - 1) * P::ns(S) + k];
    }
};

struct SyncWarp {
    __device__ __forceinline__ static void sync() { __syncwarp(); }
};
struct SyncBlock {
    __device__ __forceinline__ static void sync() { __syncthreads(); }
};

// Asynchronous global -> shared copy of one complex element (cp.async, sm_80+):
// the element is zero-filled when `valid` is false (src-size 0; the source
// address must still be a mapped one).  Completion is awaited per thread with
// cp_async_wait_all(), so a thread may read what it copied itself without a
// barrier.
template <typename T>
__device__ __forceinline__ void cp_async_elem(cpx<T>* sdst, const cpx<T>* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(cpx<T>) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 8 : 0)
                     : "memory");
    } else {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 16 : 0)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// shared-memory maps of a line's positions
template <int E>
struct RowMap {  // one row per line, one pad element every E
    int base;
    __device__ __forceinline__ int operator()(int p) const { return base + p + p / E; }
};
template <int TX>
struct ColMap {  // tile column l, position p at row p
    int l;
    __device__ __forceinline__ int operator()(int p) const { return p * TX + l; }
};

template <int L, int E, int S, int SIGN, class Sync, typename T, class Map, class Tw>
__device__ __forceinline__ void cstage(cpx<T> (&v)[E], int t, cpx<T>* sm, const Map& map, const Tw& tw) {
    using P = CPlan<L, E>;
    constexpr int R = P::radix(S), NS = P::ns(S), Q = E / R, TPL = P::TPL;
    constexpr bool LAST = S == P::NST - 1;
    SFor<0, Q>::run([&](auto ic) {
        constexpr int I = decltype(ic)::value;
        const int b = t + TPL * I;
        const int k = b & (NS - 1);
        cpx<T> a[R];
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = v[I + Q * r];
        if constexpr (S > 0) {
            SFor<1, R>::run([&](auto rc) {
                constexpr int RI = decltype(rc)::value;
                a[RI] = cmul_s<SIGN>(a[RI], tw.template get<S, I, RI>(k));
            });
        }
        dftR<R, SIGN>(a);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[I + Q * r] = a[r];
        } else {
            const int base = (b - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm[map(base + r * NS)] = a[r];
        }
    });
    if constexpr (!LAST) {
        Sync::sync();
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = sm[map(t + TPL * m)];
        Sync::sync();
    }
}

// Length-L transform of the E register elements of every thread of a line.
// Every thread of the sync scope must call it (it synchronises); the map's
// shared memory must be free.
template <int L, int E, int SIGN, class Sync, typename T, class Map, class Tw>
__device__ __forceinline__ void cfft(cpx<T> (&v)[E], int t, cpx<T>* sm, const Map& map, const Tw& tw) {
    SFor<0, CPlan<L, E>::NST>::run(
        [&](auto sc) { cstage<L, E, decltype(sc)::value, SIGN, Sync>(v, t, sm, map, tw); });
}

// ----------------------------------------------------------------------------
// Shapes per grid size and precision
// ----------------------------------------------------------------------------
template <int N, typename T>
struct CShape {
    static constexpr int L = N / 2;  // x lines: half-length complex transform
    // x pass: elements per thread (a line stays within one warp)
    static constexpr int EX = sizeof(T) == 4 ? (L >= 256 ? 16 : (L >= 64 ? 8 : 4)) : (L >= 512 ? 16 : (L >= 64 ? 8 : 4));
    static constexpr int TPLX = L / EX;
    // x pass twiddles: registers in FP32; a shared-memory table in FP64,
    // where the registers are needed for the data
    static constexpr bool XTW_REG = sizeof(T) == 4;
    static constexpr int XLPB = 256 / TPLX;  // lines per x block
    // row pitch: one pad element every EX; with two FP32 lines per warp the
    // second line's row starts half the banks away
    static constexpr int XPITCH = L + L / EX + (sizeof(T) == 4 && TPLX == 16 ? 8 : 0);
    static constexpr size_t XSMEM = ((size_t)XLPB * XPITCH + (XTW_REG ? 0 : L)) * sizeof(cpx<T>);
    // y/z passes: tile rows of TX columns (64 or 128 bytes)
    static constexpr int TX = sizeof(T) == 4 ? (N >= 512 ? 8 : 16) : (N >= 1024 ? 4 : 8);
    static constexpr int EY = sizeof(T) == 4 ? (N >= 256 ? 16 : (N >= 128 ? 8 : 4)) : (N >= 1024 ? 16 : (N >= 128 ? 8 : 4));
    static constexpr int TPLY = N / EY;
    static constexpr int YTHREADS = TX * TPLY;
    static_assert(TPLX <= 32 && 32 % TPLX == 0, "x line within a warp");
    static_assert(YTHREADS % 32 == 0 && YTHREADS <= 512, "y/z block");
};

// y/z tile shape, variant V of (N, T).  V = 0 is the default of CShape; V = 1
// and V = 2 are the alternatives the engine's autotuner times at start-up
// (FP32: 8 elements per thread, or 16-column tiles; FP64: 16 elements per
// thread, or 4-column tiles).  `valid` is false for a variant that does not
// fit a block or repeats V = 0; such variants are never instantiated.
template <int N, typename T, int V>
struct YShape {
    static constexpr bool F32 = sizeof(T) == 4;
    // V: 0 default; 1 the other element count; 2 the other tile width;
    // 3 and 4 as 0 and 1 with the stage twiddles held in registers;
    // 5 and 6 column-per-warp (CW): one warp transforms one column, 32
    // threads x N/32 elements, tiles of 8 or 16 (FP32) / 4 or 2 (FP64) columns;
    // 7 the shape of 0 compiled for three resident blocks (fewer registers,
    // more warps to hide latency)
    static constexpr bool CW = V == 5 || V == 6;
    static constexpr bool MB3 = V == 7;
    // 8: column pairs (FP32 only; ypass_pair_kernel, zfwd_pair_kernel,
    // zinv_multi_pair_kernel, PairShape), two resident blocks per SM;
    // 9: the same compiled for three (fewer registers, more warps in flight)
    static constexpr bool PAIR = V == 8 || V == 9;
    static constexpr int PAIR_MINB = V == 9 ? 3 : 2;
    static constexpr int VB = (CW || MB3) ? 0 : (V >= 3 ? V - 3 : V);
    static constexpr int EY = CW ? N / 32 : (VB == 0 ? CShape<N, T>::EY : (VB == 1 ? (F32 ? 8 : 16) : (F32 ? 16 : 8)));
    static constexpr int TX = CW ? (V == 5 ? (F32 ? 8 : 4) : (F32 ? 16 : 2))
                                 : (VB == 0 ? CShape<N, T>::TX : (VB == 1 ? 8 : (F32 ? 16 : 4)));
    static constexpr bool TWREG = V == 3 || V == 4;
    static constexpr int TPLY = N / EY;
    static constexpr int YTHREADS = TX * TPLY;
    // CW: the per-warp exchange row (one pad element every EY)
    static constexpr int WPITCH = N + N / EY;
    // two tiles (the staged next item, and the current item's exchange
    // buffer) + the twiddle table; the z stage adds the K table.  CW adds
    // the warps' exchange rows and uses two tiles in every pass.
    static constexpr size_t YSMEM =
        ((size_t)2 * N * TX + (CW ? (size_t)TX * WPITCH : 0) + N) * sizeof(cpx<T>);
    static constexpr size_t ZSMEM = YSMEM + 2 * N * sizeof(T);
    static constexpr size_t ZISMEM =
        CW ? ZSMEM : ((size_t)N * TX + N) * sizeof(cpx<T>) + 2 * N * sizeof(T);  // z inverse: one tile
    // resident blocks the register budget aims at (8 elements per thread in
    // FP32 leave room for two 512-thread blocks: 64 registers); CW: as many
    // blocks as the shared memory holds, keeping at least 96 registers
    static constexpr int CW_SMB = (int)((228 * 1024) / (ZSMEM + 1024));
    static constexpr int CW_RGB = 65536 / (YTHREADS * 96);
    static constexpr int CW_MINB = CW_SMB < CW_RGB ? CW_SMB : CW_RGB;
    static constexpr int YMINB = CW ? (CW_MINB < 1 ? 1 : CW_MINB)
                                    : MB3 ? 3 : (TWREG ? 1 : (YTHREADS <= 256 ? 2 : (F32 && EY <= 8 ? 2 : 1)));
    static constexpr bool valid =
        V == 0 || (PAIR ? (F32 && N >= 256 && N <= (V == 9 ? 512 : 1024)) :
        (MB3 ? (N >= 256 && YTHREADS <= 256 && 3 * (ZSMEM + 1024) <= 228 * 1024) :
         CW ? (N >= 256 && EY >= 2 && EY <= 16 && YTHREADS % 32 == 0 && YTHREADS <= 512 && ZSMEM <= 227 * 1024)
            : (N >= 256 && TPLY >= 2 && YTHREADS % 32 == 0 && YTHREADS <= 512 && ZSMEM <= 200 * 1024 &&
               (V >= 3 || EY != CShape<N, T>::EY || TX != CShape<N, T>::TX) && (V != 4 || F32))));
    static_assert(V != 0 || ZSMEM <= 200 * 1024, "default y/z tile fits the shared-memory limit");
};

// Column tile of TX columns x N rows for the CW variants: rows of TX
// elements, the column index XOR-swizzled by the row so that a warp reading
// one column (32 consecutive rows) and the staging threads writing whole rows
// both hit distinct banks.
template <int TX, typename T>
struct TileMap {
    static constexpr int W = (int)sizeof(cpx<T>) / 4;            // 32-bit words per element
    static constexpr int R = TX * W >= 32 ? 1 : 32 / (TX * W);   // rows per bank period
    __device__ __forceinline__ static int at(int p, int l) { return p * TX + (l ^ ((p / R) & (TX - 1))); }
};

// stage twiddles of a y/z column thread: a broadcast shared table, or registers
template <int N, int E, typename T, bool REG>
struct YTw;
template <int N, int E, typename T>
struct YTw<N, E, T, false> : TwTab<N, E, T> {
    __device__ __forceinline__ YTw(const cpx<T>* stw, const cpx<T>*, int) { this->tab = stw; }
};
template <int N, int E, typename T>
struct YTw<N, E, T, true> : TwReg<N, E, T> {
    __device__ __forceinline__ YTw(const cpx<T>*, const cpx<T>* __restrict__ gtab, int t) { this->load(gtab, t); }
};

// block-wide deterministic reduction of NR accumulators into partials[slot]
template <int NR>
__device__ __forceinline__ void block_reduce_to(const double* acc, double* out) {
    __shared__ double red_sm[32][NR];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double v = acc[r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red_sm[warp][r] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double v = lane < nw ? red_sm[lane][r] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[r] = v;
        }
    }
}

// ----------------------------------------------------------------------------
// x stage, inverse (c2r).  grid = (G, narr), block = 256.  Each block walks
// groups of 256/TPL lines of array blockIdx.y.
// ----------------------------------------------------------------------------
template <int N, typename T>
__global__ void __launch_bounds__(256, 2)
    xinv_c_kernel(XInvArgs<T> a, const cpx<T>* __restrict__ twL, const cpx<T>* __restrict__ twN) {
    using S = CShape<N, T>;
    constexpr int L = S::L, E = S::EX, TPL = S::TPLX, LPB = S::XLPB, PITCH = S::XPITCH;
    const long NG = a.nlines / LPB;  // line groups per array
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);  // LPB * PITCH, then the table
    const int ls = threadIdx.x / TPL, t = threadIdx.x % TPL;
    const RowMap<E> map{ls * PITCH};
    std::conditional_t<S::XTW_REG, TwReg<L, E, T>, TwTab<L, E, T>> tw;
    if constexpr (S::XTW_REG) {
        tw.load(twL, t);
    } else {
        cpx<T>* stw = sm + LPB * PITCH;
        for (int i = threadIdx.x; i < L; i += blockDim.x) stw[i] = twL[i];
        __syncthreads();
        tw.tab = stw;
    }
    const cpx<T> wt = twN[t];  // W_N^t
    const int nx_in = a.nx_in;
    const int px = a.px ? a.px : nx_in;  // row pitch of xs
    const cpx<T>* __restrict__ src0 = a.in[blockIdx.y];
    T* __restrict__ dst0 = a.out[blockIdx.y];
    const int src_lane = (TPL - t) & (TPL - 1);
    for (long g = blockIdx.x; g < NG; g += gridDim.x) {
        const long line = g * LPB + ls;
        const cpx<T>* __restrict__ src = src0 + line * px;
        cpx<T> v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int k = t + TPL * m;
            v[m] = k < nx_in ? src[k] : czero<T>();
        }
        // c2c + REAL() keeps the Hermitian part: real part only on kx = 0, N/2
        cpx<T> xh = czero<T>();
        if (t == 0) {
            v[0].y = T(0);
            if (L < nx_in) xh = mk(src[L].x, T(0));
        }
        cpx<T> o[E];
        SFor<0, E>::run([&](auto mc) {
            constexpr int m = decltype(mc)::value;
            cpx<T> xp;  // X[L - k], k = t + TPL m
            xp.x = __shfl_sync(0xffffffffu, v[E - 1 - m].x, src_lane, TPL);
            xp.y = __shfl_sync(0xffffffffu, v[E - 1 - m].y, src_lane, TPL);
            if (t == 0) xp = (m == 0) ? xh : v[(E - m) % E];
            const cpx<T> xk = v[m];
            const cpx<T> xc = conj(xp);
            const cpx<T> Fk = xk + xc;
            // G = (xk - xc) * conj(W_N^k),  W_N^k = W_N^t * W_N^(TPL m)
            const cpx<T> w = wt * cw<T, N, (long)TPL * m>();
            const cpx<T> G = cmul_s<+1>(xk - xc, w);
            o[m] = mk(Fk.x - G.y, Fk.y + G.x);  // F + i G
        });
        cfft<L, E, +1, SyncWarp>(o, t, sm, map, tw);
        cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(dst0 + line * N);
#pragma unroll
        for (int m = 0; m < E; ++m) dst[t + TPL * m] = o[m];
    }
}

// ----------------------------------------------------------------------------
// x stage, forward: functor on the physical inputs, then the real FFT of each
// functor output along x (a complex transform of length N/2 of the packed
// pairs, then the half-spectrum split).  grid = G, block = 256: each block
// walks groups of 256/TPL lines; output 0 stays in registers, outputs 1.. are
// parked in thread-private shared-memory slots until their turn.
// ----------------------------------------------------------------------------
template <int N, typename T, int NOUT>
struct XFwdSmem {
    using S = CShape<N, T>;
    static constexpr size_t STAGE = (size_t)(NOUT > 1 ? NOUT - 1 : 0) * S::XLPB * S::L;
    static constexpr size_t BYTES = (STAGE + (size_t)S::XLPB * S::XPITCH + (S::XTW_REG ? 0 : S::L)) * sizeof(cpx<T>);
};

// positions whose inputs are loaded together: about 32 loads per thread
__host__ __device__ constexpr int xfwd_chunk(int nin, int e) {
    int c = 1;
    while (2 * c <= e && 2 * c * nin <= 32) c *= 2;
    return c;
}

// resident blocks the register budget aims at: light functors 2, heavy ones 1
template <class F>
constexpr int xfwd_minb() {
    return F::NIN + F::NOUT <= 8 ? 2 : 1;
}

template <int N, typename T, class F>
__global__ void __launch_bounds__(256, xfwd_minb<F>())
    xfwd_c_kernel(XFwdArgs<T> a, F f, const cpx<T>* __restrict__ twL, const cpx<T>* __restrict__ twN) {
    using S = CShape<N, T>;
    constexpr int NIN = F::NIN, NOUT = F::NOUT, NR = F::NRED;
    constexpr int L = S::L, E = S::EX, TPL = S::TPLX, LPB = S::XLPB, PITCH = S::XPITCH;
    constexpr int CHX = xfwd_chunk(NIN, E);
    const long NG = a.nlines / LPB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* stg = reinterpret_cast<cpx<T>*>(smem_raw);              // [NOUT-1][LPB][L]
    cpx<T>* sm = stg + XFwdSmem<N, T, NOUT>::STAGE;                  // [LPB][PITCH]
    const int ls = threadIdx.x / TPL, t = threadIdx.x % TPL;
    const RowMap<E> map{ls * PITCH};
    std::conditional_t<S::XTW_REG, TwReg<L, E, T>, TwTab<L, E, T>> tw;
    if constexpr (S::XTW_REG) {
        tw.load(twL, t);
    } else {
        cpx<T>* stw = sm + LPB * PITCH;
        for (int i = threadIdx.x; i < L; i += blockDim.x) stw[i] = twL[i];
        __syncthreads();
        tw.tab = stw;
    }
    const cpx<T> wt = twN[t];  // W_N^t
    const int nx = a.nx;
    const int px = a.px ? a.px : nx;  // row pitch of xs
    const int src_lane = (TPL - t) & (TPL - 1);
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    for (long g = blockIdx.x; g < NG; g += gridDim.x) {
        const long line = g * LPB + ls;
        // 1. functor on the pairs (2p, 2p+1), p = t + TPL m.  The inputs of CHX
        // positions are loaded before the functor runs on any of them, so
        // CHX * NIN loads per thread are in flight.
        cpx<T> v[E];
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += CHX) {
            cpx<T> ld[CHX][NIN];
#pragma unroll
            for (int j = 0; j < CHX; ++j)
#pragma unroll
                for (int i = 0; i < NIN; ++i)
                    ld[j][i] = *reinterpret_cast<const cpx<T>*>(a.in[i] + line * N + 2 * (t + TPL * (m0 + j)));
#pragma unroll
            for (int j = 0; j < CHX; ++j) {
                const int p = t + TPL * (m0 + j);
                T in0[NIN], in1[NIN];
#pragma unroll
                for (int i = 0; i < NIN; ++i) {
                    in0[i] = ld[j][i].x;
                    in1[i] = ld[j][i].y;
                }
                T o0[NOUT > 0 ? NOUT : 1], o1[NOUT > 0 ? NOUT : 1];
                f(in0, o0, acc);
                f(in1, o1, acc);
                v[m0 + j] = mk(o0[0], o1[0]);
#pragma unroll
                for (int o = 1; o < NOUT; ++o) stg[((o - 1) * LPB + ls) * L + p] = mk(o0[o], o1[o]);
            }
        }
        // 2. per output: complex FFT of the packed row, half-spectrum split
#pragma unroll 1
        for (int o = 0; o < NOUT; ++o) {
            if (o > 0) {
#pragma unroll
                for (int m = 0; m < E; ++m) v[m] = stg[((o - 1) * LPB + ls) * L + t + TPL * m];
            }
            cfft<L, E, -1, SyncWarp>(v, t, sm, map, tw);
            if (t == 0 && a.nanflag && !cpx_finite(v[0])) *a.nanflag = 1.0;  // the DC bin of the line
            cpx<T>* __restrict__ dst = a.out[o] + line * px;
            // X[k] = E[k] + W_N^k O[k], E = (Z_k + conj Z_{L-k})/2, O = -i (Z_k - conj Z_{L-k})/2
            SFor<0, E>::run([&](auto mc) {
                constexpr int m = decltype(mc)::value;
                cpx<T> zp;  // Z[(L - k) mod L], k = t + TPL m
                zp.x = __shfl_sync(0xffffffffu, v[E - 1 - m].x, src_lane, TPL);
                zp.y = __shfl_sync(0xffffffffu, v[E - 1 - m].y, src_lane, TPL);
                if (t == 0) zp = v[(E - m) % E];
                const int k = t + TPL * m;
                const cpx<T> zc = conj(zp);
                const cpx<T> Ev = (v[m] + zc) * T(0.5);
                const cpx<T> D = (v[m] - zc) * T(0.5);
                const cpx<T> O = mk(D.y, -D.x);
                const cpx<T> w = wt * cw<T, N, (long)TPL * m>();
                if (k < nx) dst[k] = Ev + O * w;
            });
            // Nyquist column (full band only): X[N/2] = Re Z0 - Im Z0
            if (t == 0 && L < nx) dst[L] = mk(v[0].x - v[0].y, T(0));
            if (t == 0 && nx < px) dst[nx] = czero<T>();  // the pitch's pad column stays zero
            __syncwarp();
        }
    }
    if constexpr (NR > 0) block_reduce_store<NR>(acc, a.partials, blockIdx.x);
}

// ----------------------------------------------------------------------------
// y pass.  grid = (G, narr), block = TX * TPLY.  Items: (z, kx tile).
// ----------------------------------------------------------------------------
template <int N, int V, int SIGN, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    ypass_c_kernel(YArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    constexpr int E = S::EY, TPL = S::TPLY, TX = S::TX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* buf0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* buf1 = buf0 + N * TX;
    cpx<T>* stw = buf1 + N * TX;
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    __syncthreads();
    const int l = threadIdx.x % TX, t = threadIdx.x / TX;
    const YTw<N, E, T, S::TWREG> tw(stw, twN, t);
    const ColMap<TX> map{l};
    const int nx = a.nx, nb = a.band.nb;
    const int px = a.px ? a.px : nx;  // row pitch of xs and ys
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)a.nz * ntile;
    const cpx<T>* __restrict__ src = a.in[blockIdx.y];
    cpx<T>* __restrict__ dst = a.out[blockIdx.y];
    // stage item `it` (column tile of plane z) into buffer b, asynchronously
    auto stage = [&](long it, cpx<T>* b) {
        const int z = (int)(it / ntile);
        const int kx = (int)(it - (long)z * ntile) * TX + l;
        const bool ok = kx < nx;
        const int kxc = ok ? kx : nx - 1;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int p = t + TPL * m;
            if constexpr (SIGN < 0) {
                cp_async_elem(b + p * TX + l, src + ((long)z * N + p) * px + kxc, ok);
            } else {
                const int ci = band_compact_index(a.band, p);
                cp_async_elem(b + p * TX + l, src + ((long)z * nb + (ci >= 0 ? ci : 0)) * px + kxc, ok && ci >= 0);
            }
        }
        cp_async_commit();
    };
    long it = blockIdx.x;
    if (it < items) stage(it, buf0);
    for (int k = 0; it < items; it += gridDim.x, k ^= 1) {
        cpx<T>* cur = k ? buf1 : buf0;
        cpx<T>* nxt = k ? buf0 : buf1;
        cp_async_wait_all();
        cpx<T> v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = cur[map(t + TPL * m)];
        // every thread has its tile in registers and the previous transform is
        // done: cur becomes this transform's exchange buffer, nxt the next stage
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        cfft<N, E, SIGN, SyncBlock>(v, t, cur, map, tw);
        const int z = (int)(it / ntile);
        const int kx = (int)(it - (long)z * ntile) * TX + l;
        if (kx < nx) {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int p = t + TPL * m;
                if constexpr (SIGN < 0) {
                    const int ci = band_compact_index(a.band, p);
                    if (ci >= 0) dst[((long)z * nb + ci) * px + kx] = v[m];
                } else {
                    dst[((long)z * N + p) * px + kx] = v[m];
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Spectral symbols in the pipeline precision C.  The wavenumbers come from a
// per-block table K[f] = 2 pi j(f) (and its odd-factor copy, 0 at the Nyquist
// index), built exactly as make_k does; with C = double every symbol is the
// same arithmetic as apply_sym.  With C = float (mixed mode) the multiply by
// the symbol rounds like the FP32 transforms around it; reductions stay FP64.
// ----------------------------------------------------------------------------
template <typename C>
__device__ __forceinline__ cpx<C> ld_spec_c(const void* p, int f64, long idx) {
    if (f64) {
        const double2 v = reinterpret_cast<const double2*>(p)[idx];
        return mk((C)v.x, (C)v.y);
    }
    const float2 v = reinterpret_cast<const float2*>(p)[idx];
    return mk((C)v.x, (C)v.y);
}
template <typename C>
__device__ __forceinline__ void st_spec_c(void* p, int f64, long idx, cpx<C> v) {
    if (f64)
        reinterpret_cast<double2*>(p)[idx] = make_double2((double)v.x, (double)v.y);
    else
        reinterpret_cast<float2*>(p)[idx] = make_float2((float)v.x, (float)v.y);
}

// A spectral symbol times a coefficient in branch-free form:
//   f(k) = c1 + ck o_a + cq |K|^2 + (ci + ckk o_a o_b) / |K|^2   (last term 0 at K = 0)
// applied as f v, or i f v for the odd (first-derivative) symbols.  Every Sym
// is a special case; the per-element work is a few selects and FMAs instead
// of a switch.
template <typename C>
struct SymD {
    C c1, ck, cq, ci, ckk;
    int a, b;
    bool odd, inv;
};
template <typename C>
__device__ __forceinline__ SymD<C> make_symd(int sym, int ab, double coef) {
    SymD<C> d{C(0), C(0), C(0), C(0), C(0), 0, 0, false, false};
    const C c = (C)coef;
    switch (sym) {
        case SYM_ONE: d.c1 = c; break;
        case SYM_IKX: d.ck = c; d.a = 0; d.odd = true; break;
        case SYM_IKY: d.ck = c; d.a = 1; d.odd = true; break;
        case SYM_IKZ: d.ck = c; d.a = 2; d.odd = true; break;
        case SYM_NEG_KSQ: d.cq = -c; break;
        case SYM_INV_KSQ: d.ci = c; d.inv = true; break;
        case SYM_NEG_INV_KSQ: d.ci = -c; d.inv = true; break;
        case SYM_KK_KSQ: d.ckk = c; d.a = ab / 3; d.b = ab % 3; d.inv = true; break;
        default: break;  // SYM_ZERO: f = 0
    }
    return d;
}
// rinv = 1/|K|^2 (0 at K = 0), needed only when d.inv
template <typename C>
__device__ __forceinline__ cpx<C> sym_apply(const SymD<C>& d, C ox, C oy, C oz, C ksq, C rinv, cpx<C> v) {
    const C oa = d.a == 0 ? ox : (d.a == 1 ? oy : oz);
    C f = d.c1 + d.ck * oa + d.cq * ksq;
    if (d.inv) {
        const C ob = d.b == 0 ? ox : (d.b == 1 ? oy : oz);
        f += rinv * (d.ci + d.ckk * oa * ob);
    }
    return d.odd ? mk(-f * v.y, f * v.x) : mk(f * v.x, f * v.y);
}
template <typename C>
__device__ __forceinline__ C rinv_of(C ksq) {
    return ksq == C(0) ? C(0) : C(1) / ksq;
}

// K table (2 pi j, then the odd-factor copy) of length 2N in shared memory
template <int N, typename C>
__device__ __forceinline__ void fill_k_table(C* kt) {
    const double twopi = 2.0 * 3.14159265358979311600;  // 2.0_pr*PI, PI = 4 atan2(1,1)
    for (int f = threadIdx.x; f < N; f += blockDim.x) {
        const double K = twopi * (double)signed_j(N, f);
        kt[f] = (C)K;
        kt[N + f] = (f == N / 2) ? C(0) : (C)K;
    }
}

// Batched spectrum loads: CH elements m0..m0+CH-1 of a column, every load
// issued before any is used (indices are clamped in bounds, so no load sits
// behind a per-element branch and CH loads per thread are in flight).
template <int CH, typename C, class Idx>
__device__ __forceinline__ void ld_chunk(const void* p, int f64, const Idx& idx, int m0, cpx<C> (&out)[CH]) {
    if (f64) {
        const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const double2 v = q[idx(m0 + j)];
            out[j] = mk((C)v.x, (C)v.y);
        }
    } else {
        const float2* q = reinterpret_cast<const float2*>(p);
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const float2 v = q[idx(m0 + j)];
            out[j] = mk((C)v.x, (C)v.y);
        }
    }
}

// Column geometry of a z-stage item: compact z index of FFT position
// t + TPL m, validity and the (clamped, in-bounds) spectrum index.
template <int N, int TPL>
struct ZCol {
    int t, cut, nb, plane, col;
    bool ok;
    __device__ __forceinline__ int cz(int m) const {
        const int fz = t + TPL * m;
        return fz <= cut ? fz : (fz >= N - cut ? fz - (N - nb) : -1);
    }
    __device__ __forceinline__ bool valid(int m) const { return ok && cz(m) >= 0; }
    __device__ __forceinline__ int operator()(int m) const {
        const int c = cz(m);
        return (c >= 0 ? c : 0) * plane + col;
    }
};

// Spectral side of a z-forward item, on the column elements Y[m] (z position
// t + TPL m, forward-transformed): the main symbol (the 1/N^3 folded in), the
// optional added term, the reductions and the optional pruned-spectrum store.
// Y is left holding the spectrum (zero outside the band).
struct ZAcc {
    double self = 0.0, w[3] = {0.0, 0.0, 0.0};
};
template <int N, int E, int TPL, typename C>
__device__ __forceinline__ void zfwd_spectral(const ZFwdOp& op, const SymD<C>& dmain, const SymD<C>& dadd,
                                              const C* kt, const ZCol<N, TPL>& idx, int fy, int kxc, double wgt,
                                              cpx<C> (&Y)[E], ZAcc& acc) {
    constexpr int CH = E < 8 ? E : 8;
    const C ox = kt[N + kxc], oy = kt[N + fy];
    const C kxy2 = kt[kxc] * kt[kxc] + kt[fy] * kt[fy];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int fz = idx.t + TPL * m;
        const C kz = kt[fz], oz = kt[N + fz];
        const C ksq = kxy2 + kz * kz;
        const C ri = dmain.inv ? rinv_of(ksq) : C(0);
        Y[m] = idx.valid(m) ? sym_apply(dmain, ox, oy, oz, ksq, ri, Y[m]) : mk(C(0), C(0));
    }
    if (op.add) {
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += CH) {
            cpx<C> A[CH];
            ld_chunk<CH>(op.add, op.add_f64, idx, m0, A);
#pragma unroll
            for (int j = 0; j < CH; ++j) {
                const int fz = idx.t + TPL * (m0 + j);
                const C kz = kt[fz], oz = kt[N + fz];
                const C ksq = kxy2 + kz * kz;
                const C ri = dadd.inv ? rinv_of(ksq) : C(0);
                if (idx.valid(m0 + j)) Y[m0 + j] = Y[m0 + j] + sym_apply(dadd, ox, oy, oz, ksq, ri, A[j]);
            }
        }
    }
    if (op.red_self >= 0) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const double yx = (double)Y[m].x, yy = (double)Y[m].y;
            acc.self += wgt * (yx * yx + yy * yy);  // zero outside the band
        }
    }
#pragma unroll 1
    for (int r = 0; r < 3; ++r) {
        if (!op.red_with[r]) continue;
        double s = 0.0;
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += CH) {
            cpx<double> W[CH];
            ld_chunk<CH>(op.red_with[r], op.red_with_f64[r], idx, m0, W);
#pragma unroll
            for (int j = 0; j < CH; ++j) s += (double)Y[m0 + j].x * W[j].x + (double)Y[m0 + j].y * W[j].y;
        }
        acc.w[r] += wgt * s;
    }
    if (op.spec_out) {
#pragma unroll
        for (int m = 0; m < E; ++m)
            if (idx.valid(m)) st_spec_c(op.spec_out, op.spec_f64, idx(m), Y[m]);
    }
}

// The spectral side of a column-pair item (kx = 2 pr and 2 pr + 1 of row cy):
// what two zfwd_spectral calls (column 0, then column 1) do, with the row
// tests, the z wavenumbers and the row offsets computed once for both
// columns, and both columns stored as one 16-byte vector where the pair is
// aligned in an FP32 spectrum.  The reductions add column 0's terms before
// column 1's in the same order, so the sums are those of the two calls.
template <int N, int E, int TPL>
__device__ __forceinline__ void zfwd_spectral_pair(const ZFwdOp& op, const SymD<float>& dmain,
                                                   const SymD<float>& dadd, const float* kt, int t, int cut, int nb,
                                                   int plane, int nx, int cy, int pr, int fy, cpx<float> (&Ya)[E],
                                                   cpx<float> (&Yb)[E], ZAcc& acc) {
    using C = float;
    const int kx0 = 2 * pr, kx1 = 2 * pr + 1;
    const bool ok0 = kx0 < nx, ok1 = kx1 < nx;
    const int kc0 = ok0 ? kx0 : nx - 1, kc1 = ok1 ? kx1 : nx - 1;  // clamped: loads stay in bounds
    const int col0 = cy * nx + kc0, col1 = cy * nx + kc1;
    const C oy = kt[N + fy], ky2 = kt[fy] * kt[fy];
    const C ox0 = kt[N + kc0], ox1 = kt[N + kc1];
    const C kxy0 = kt[kc0] * kt[kc0] + ky2, kxy1 = kt[kc1] * kt[kc1] + ky2;
    int roff[E];
    bool rv[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int fz = t + TPL * m;
        const int cz = fz <= cut ? fz : (fz >= N - cut ? fz - (N - nb) : -1);
        rv[m] = cz >= 0;
        roff[m] = (cz >= 0 ? cz : 0) * plane;
    }
    // main symbol (the 1/N^3 folded in) and the optional added term
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int fz = t + TPL * m;
        const C kz = kt[fz], oz = kt[N + fz], kz2 = kz * kz;
        const C ksq0 = kxy0 + kz2, ksq1 = kxy1 + kz2;
        const C ri0 = dmain.inv ? rinv_of(ksq0) : C(0), ri1 = dmain.inv ? rinv_of(ksq1) : C(0);
        Ya[m] = (rv[m] && ok0) ? sym_apply(dmain, ox0, oy, oz, ksq0, ri0, Ya[m]) : mk(C(0), C(0));
        Yb[m] = (rv[m] && ok1) ? sym_apply(dmain, ox1, oy, oz, ksq1, ri1, Yb[m]) : mk(C(0), C(0));
    }
    if (op.add) {
        cpx<C> A0[E], A1[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            A0[m] = ld_spec_c<C>(op.add, op.add_f64, (long)roff[m] + col0);
            A1[m] = ld_spec_c<C>(op.add, op.add_f64, (long)roff[m] + col1);
        }
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int fz = t + TPL * m;
            const C kz = kt[fz], oz = kt[N + fz], kz2 = kz * kz;
            const C ksq0 = kxy0 + kz2, ksq1 = kxy1 + kz2;
            const C ri0 = dadd.inv ? rinv_of(ksq0) : C(0), ri1 = dadd.inv ? rinv_of(ksq1) : C(0);
            if (rv[m] && ok0) Ya[m] = Ya[m] + sym_apply(dadd, ox0, oy, oz, ksq0, ri0, A0[m]);
            if (rv[m] && ok1) Yb[m] = Yb[m] + sym_apply(dadd, ox1, oy, oz, ksq1, ri1, A1[m]);
        }
    }
    const double w0 = kx_weight(N, kx0), w1 = kx_weight(N, kx1);
    if (op.red_self >= 0) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const double yx = (double)Ya[m].x, yy = (double)Ya[m].y;
            acc.self += w0 * (yx * yx + yy * yy);
        }
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const double yx = (double)Yb[m].x, yy = (double)Yb[m].y;
            acc.self += w1 * (yx * yx + yy * yy);
        }
    }
#pragma unroll 1
    for (int r = 0; r < 3; ++r) {
        if (!op.red_with[r]) continue;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const cpx<double> W0 = ld_spec_c<double>(op.red_with[r], op.red_with_f64[r], (long)roff[m] + col0);
            const cpx<double> W1 = ld_spec_c<double>(op.red_with[r], op.red_with_f64[r], (long)roff[m] + col1);
            s0 += (double)Ya[m].x * W0.x + (double)Ya[m].y * W0.y;
            s1 += (double)Yb[m].x * W1.x + (double)Yb[m].y * W1.y;
        }
        acc.w[r] += w0 * s0;
        acc.w[r] += w1 * s1;
    }
    if (op.spec_out) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
            if (!rv[m]) continue;
            const long e0 = (long)roff[m] + col0;
            float2* p0 = reinterpret_cast<float2*>(op.spec_out) + e0;
            // one 16-byte store only where the pair's address is 16-byte
            // aligned (array and component bases are only 8-byte aligned)
            if (!op.spec_f64 && ok0 && ok1 && (reinterpret_cast<uintptr_t>(p0) & 15) == 0) {
                *reinterpret_cast<float4*>(p0) = make_float4(Ya[m].x, Ya[m].y, Yb[m].x, Yb[m].y);
            } else {
                if (ok0) st_spec_c(op.spec_out, op.spec_f64, e0, Ya[m]);
                if (ok1) st_spec_c(op.spec_out, op.spec_f64, (long)roff[m] + col1, Yb[m]);
            }
        }
    }
}

// one reduction record of MAX_RED partials per block from the accumulators
__device__ __forceinline__ void zfwd_partials(const ZFwdOp& op, const ZAcc& acc, double* part) {
    const bool any_red = op.red_self >= 0 || op.red_with[0] || op.red_with[1] || op.red_with[2];
    if (any_red) {
        double acc4[4] = {acc.self, acc.w[0], acc.w[1], acc.w[2]};
        __shared__ double part4[4];
        block_reduce_to<4>(acc4, part4);
        __syncthreads();
        if (threadIdx.x < MAX_RED) {
            double s = 0.0;
            if ((int)threadIdx.x == op.red_self) s += part4[0];
            for (int r = 0; r < 3; ++r)
                if (op.red_with[r] && (int)threadIdx.x == op.red_with_slot[r]) s += part4[1 + r];
            part[threadIdx.x] = s;
        }
    } else if (threadIdx.x < MAX_RED) {
        part[threadIdx.x] = 0.0;
    }
}

// ----------------------------------------------------------------------------
// z stage, forward (+ optional round trip).  grid = (G, narr); items (cy, tile).
// One reduction record of MAX_RED partials per block.
// ----------------------------------------------------------------------------
template <int N, int V, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    zfwd_c_kernel(ZFwdArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using C = T;
    constexpr int E = S::EY, TPL = S::TPLY, TX = S::TX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* buf0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* buf1 = buf0 + N * TX;
    cpx<T>* stw = buf1 + N * TX;
    C* kt = reinterpret_cast<C*>(stw + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    fill_k_table<N>(kt);
    __syncthreads();
    const int l = threadIdx.x % TX, t = threadIdx.x / TX;
    const YTw<N, E, T, S::TWREG> tw(stw, twN, t);
    const ColMap<TX> map{l};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)nb * ntile;
    const ZFwdOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;                      // spectra
    const int px = a.px ? a.px : nx, yplane = nb * px;  // y-stage arrays
    const cpx<T>* __restrict__ src = reinterpret_cast<const cpx<T>*>(op.in);
    cpx<T>* __restrict__ yout = reinterpret_cast<cpx<T>*>(op.ys_out);
    const SymD<C> dmain = make_symd<C>(op.sym, op.sym_ab, a.norm);  // the 1/N^3 folded in
    const SymD<C> dadd = make_symd<C>(op.add_sym, op.add_ab, op.add_coef);
    ZAcc acc;
    // stage the ys column tile of item `it` into buffer b, asynchronously
    auto stage = [&](long it, cpx<T>* b) {
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + l;
        const bool ok = kx < nx;
        const int ycol = cy * px + (ok ? kx : nx - 1);
#pragma unroll
        for (int m = 0; m < E; ++m) cp_async_elem(b + (t + TPL * m) * TX + l, src + (t + TPL * m) * yplane + ycol, ok);
        cp_async_commit();
    };
    long it0 = blockIdx.x;
    if (it0 < items) stage(it0, buf0);
    int kbuf = 0;
    for (long it = it0; it < items; it += gridDim.x, kbuf ^= 1) {
        cpx<T>* sm = kbuf ? buf1 : buf0;  // this item's tile, then its exchange buffer
        cpx<T>* nxt = kbuf ? buf0 : buf1;
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + l;
        const bool ok = kx < nx;
        const int col = cy * nx + (ok ? kx : nx - 1);  // clamped: loads stay in bounds
        cp_async_wait_all();
        cpx<T> v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = sm[map(t + TPL * m)];
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        cfft<N, E, -1, SyncBlock>(v, t, sm, map, tw);
        const int fy = band_fft_index(a.band, cy);
        const int kxc = col - cy * nx;
        const ZCol<N, TPL> idx{t, cut, nb, plane, col, ok};
        cpx<C> Y[E];
#pragma unroll
        for (int m = 0; m < E; ++m) Y[m] = mk((C)v[m].x, (C)v[m].y);
        zfwd_spectral<N, E, TPL>(op, dmain, dadd, kt, idx, fy, kxc, kx_weight(N, kx), Y, acc);
        if (yout) {
#pragma unroll
            for (int m = 0; m < E; ++m) v[m] = mk((T)Y[m].x, (T)Y[m].y);
            cfft<N, E, +1, SyncBlock>(v, t, sm, map, tw);
            if (ok) {
#pragma unroll
                for (int m = 0; m < E; ++m) yout[(t + TPL * m) * yplane + cy * px + kx] = v[m];
            }
        }
    }
    zfwd_partials(op, acc, a.partials + (long)(blockIdx.y * gridDim.x + blockIdx.x) * MAX_RED);
}

// ----------------------------------------------------------------------------
// z stage, inverse from spectra.  grid = (G, narr); items (cy, tile).
// ----------------------------------------------------------------------------
template <int N, int V, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    zinv_c_kernel(ZInvArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using C = T;
    constexpr int E = S::EY, TPL = S::TPLY, TX = S::TX, CH = E < 8 ? E : 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* stw = sm + N * TX;
    C* kt = reinterpret_cast<C*>(stw + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    fill_k_table<N>(kt);
    __syncthreads();
    const int l = threadIdx.x % TX, t = threadIdx.x / TX;
    const YTw<N, E, T, S::TWREG> tw(stw, twN, t);
    const ColMap<TX> map{l};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)nb * ntile;
    const ZInvOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;                      // spectra
    const int px = a.px ? a.px : nx, yplane = nb * px;  // y-stage arrays
    const int nsrc = op.nsrc;
    cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(op.ys_out);
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + l;
        const bool ok = kx < nx;
        const int col = cy * nx + (ok ? kx : nx - 1);  // clamped: loads stay in bounds
        const int fy = band_fft_index(a.band, cy);
        const int kxc = col - cy * nx;
        const C kxv = kt[kxc], ox = kt[N + kxc], kyv = kt[fy], oy = kt[N + fy];
        const C kxy2 = kxv * kxv + kyv * kyv;
        const ZCol<N, TPL> idx{t, cut, nb, plane, col, ok};
        cpx<C> Y[E];
#pragma unroll
        for (int m = 0; m < E; ++m) Y[m] = mk(C(0), C(0));
#pragma unroll 1
        for (int s = 0; s < nsrc; ++s) {
            const void* spec = op.src[s].spec;
            const int f64 = op.src[s].f64;
            const SymD<C> d = make_symd<C>(op.src[s].sym, op.src[s].ab, op.src[s].coef);
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += CH) {
                cpx<C> Vv[CH];
                ld_chunk<CH>(spec, f64, idx, m0, Vv);
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int fz = t + TPL * (m0 + j);
                    const C kz = kt[fz], oz = kt[N + fz];
                    const C ksq = kxy2 + kz * kz;
                    const C ri = d.inv ? rinv_of(ksq) : C(0);
                    if (idx.valid(m0 + j)) Y[m0 + j] = Y[m0 + j] + sym_apply(d, ox, oy, oz, ksq, ri, Vv[j]);
                }
            }
        }
        cpx<T> v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = mk((T)Y[m].x, (T)Y[m].y);
        cfft<N, E, +1, SyncBlock>(v, t, sm, map, tw);
        if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) dst[(t + TPL * m) * yplane + cy * px + kx] = v[m];
        }
    }
}

// ----------------------------------------------------------------------------
// z stage, inverse, one source and up to ZMULTI outputs per op: the column of
// the source spectrum is loaded once, then each output applies its symbol,
// transforms and stores.  grid = (G, nops); the tile shape of variant V.
// ----------------------------------------------------------------------------
template <int N, int V, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    zinv_multi_c_kernel(ZInvMultiArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using C = T;
    constexpr int E = S::EY, TPL = S::TPLY, TX = S::TX, CH = E < 8 ? E : 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* stw = sm + N * TX;
    C* kt = reinterpret_cast<C*>(stw + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    fill_k_table<N>(kt);
    __syncthreads();
    const int l = threadIdx.x % TX, t = threadIdx.x / TX;
    const YTw<N, E, T, S::TWREG> tw(stw, twN, t);
    const ColMap<TX> map{l};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)nb * ntile;
    const ZInvMultiOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;                          // spectra
    const int px = a.px ? a.px : nx, yplane = nb * px;  // y-stage arrays
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + l;
        const bool ok = kx < nx;
        const int col = cy * nx + (ok ? kx : nx - 1);  // clamped: loads stay in bounds
        const int fy = band_fft_index(a.band, cy);
        const int kxc = col - cy * nx;
        const C ox = kt[N + kxc], oy = kt[N + fy];
        const C kxy2 = kt[kxc] * kt[kxc] + kt[fy] * kt[fy];
        const ZCol<N, TPL> idx{t, cut, nb, plane, col, ok};
        cpx<C> Vv[E];
#pragma unroll
        for (int m0 = 0; m0 < E; m0 += CH) {
            cpx<C> ch[CH];
            ld_chunk<CH>(op.spec, op.f64, idx, m0, ch);
#pragma unroll
            for (int j = 0; j < CH; ++j) Vv[m0 + j] = ch[j];
        }
#pragma unroll 1
        for (int o = 0; o < op.nout; ++o) {
            const SymD<C> d = make_symd<C>(op.sym[o], op.ab[o], op.coef[o]);
            cpx<T> v[E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int fz = t + TPL * m;
                const C kz = kt[fz], oz = kt[N + fz];
                const C ksq = kxy2 + kz * kz;
                const C ri = d.inv ? rinv_of(ksq) : C(0);
                const cpx<C> y = idx.valid(m) ? sym_apply(d, ox, oy, oz, ksq, ri, Vv[m]) : mk(C(0), C(0));
                v[m] = mk((T)y.x, (T)y.y);
            }
            cfft<N, E, +1, SyncBlock>(v, t, sm, map, tw);
            if (ok) {
                cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(op.ys_out[o]);
#pragma unroll
                for (int m = 0; m < E; ++m) dst[(t + TPL * m) * yplane + cy * px + kx] = v[m];
            }
        }
    }
}

// ----------------------------------------------------------------------------
// y pass on column pairs (FP32, variant V = 8 of YShape).  Each thread
// transforms the two neighbouring kx columns 2j and 2j+1 of a tile at once:
// they share every twiddle, index and address computation, and move through
// global and shared memory as one 16-byte float4 (a row pitch that is even
// keeps every pair 16-byte aligned; the pad column of an odd nx rides along
// as the second column of the last pair).  E = 8 elements per column and
// thread, radix-8 Stockham stages.  Tile: NP = 4 pairs (8 columns) x N rows
// of float4, swizzled so that the stage exchanges are free of bank conflicts.
// ----------------------------------------------------------------------------
template <int N>
struct PairShape {
    static constexpr int E = 8, NP = 4;
    static constexpr int TPL = N / E;         // threads per column pair
    static constexpr int THREADS = NP * TPL;
    static constexpr int TILE = N * NP;       // float4 slots of one tile
    static constexpr size_t SMEM = (size_t)2 * TILE * sizeof(float4) + (size_t)N * sizeof(cpx<float>);
    static_assert(THREADS % 32 == 0 && THREADS <= 512, "pair block");
};

// slot of row p, pair l: row-major, with rows 8..15 (mod 16) swapped with
// their neighbour row so that rows p and p + 8 fall in different halves of
// the 8 16-byte bank groups (16-byte accesses are served 8 threads at a time)
__device__ __forceinline__ int pair_slot(int p, int l) { return (4 * p + l) ^ (((p >> 3) & 1) << 2); }

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 16 : 0)
                 : "memory");
}

template <int L, int E, int S, int SIGN, class Tw>
__device__ __forceinline__ void pstage(cpx<float> (&va)[E], cpx<float> (&vb)[E], int t, int l, float4* sm,
                                       const Tw& tw) {
    using P = CPlan<L, E>;
    constexpr int R = P::radix(S), NS = P::ns(S), Q = E / R, TPL = P::TPL;
    constexpr bool LAST = S == P::NST - 1;
    SFor<0, Q>::run([&](auto ic) {
        constexpr int I = decltype(ic)::value;
        const int b = t + TPL * I;
        const int k = b & (NS - 1);
        cpx<float> a[R], c[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            a[r] = va[I + Q * r];
            c[r] = vb[I + Q * r];
        }
        if constexpr (S > 0) {
            SFor<1, R>::run([&](auto rc) {
                constexpr int RI = decltype(rc)::value;
                const cpx<float> w = tw.template get<S, I, RI>(k);
                a[RI] = cmul_s<SIGN>(a[RI], w);
                c[RI] = cmul_s<SIGN>(c[RI], w);
            });
        }
        dftR<R, SIGN>(a);
        dftR<R, SIGN>(c);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                va[I + Q * r] = a[r];
                vb[I + Q * r] = c[r];
            }
        } else {
            const int base = (b - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm[pair_slot(base + r * NS, l)] = make_float4(a[r].x, a[r].y, c[r].x, c[r].y);
        }
    });
    if constexpr (!LAST) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const float4 q = sm[pair_slot(t + TPL * m, l)];
            va[m] = mk(q.x, q.y);
            vb[m] = mk(q.z, q.w);
        }
        __syncthreads();
    }
}

template <int N, int SIGN, int MINB>
__global__ void __launch_bounds__(PairShape<N>::THREADS, MINB)
    ypass_pair_kernel(YArgs<float> a, const cpx<float>* __restrict__ twN) {
    using S = PairShape<N>;
    constexpr int E = S::E, TPL = S::TPL, NP = S::NP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* buf0 = reinterpret_cast<float4*>(smem_raw);
    float4* buf1 = buf0 + S::TILE;
    cpx<float>* stw = reinterpret_cast<cpx<float>*>(buf1 + S::TILE);
    TwStage<N, E, float>::fill(stw, twN);
    __syncthreads();
    const int l = threadIdx.x % NP, t = threadIdx.x / NP;
    const TwStage<N, E, float> tw{stw};
    const int nx = a.nx, nb = a.band.nb;
    const int pp = (a.px ? a.px : nx) / 2;  // row pitch in pairs (the pitch is even)
    const int npair = (nx + 1) / 2;
    const int ntile = (npair + NP - 1) / NP;
    const long items = (long)a.nz * ntile;
    const float4* __restrict__ src = reinterpret_cast<const float4*>(a.in[blockIdx.y]);
    float4* __restrict__ dst = reinterpret_cast<float4*>(a.out[blockIdx.y]);
    auto stage = [&](long it, float4* b) {
        const int z = (int)(it / ntile);
        const int pr = (int)(it - (long)z * ntile) * NP + l;
        const bool ok = pr < npair;
        const int prc = ok ? pr : npair - 1;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int p = t + TPL * m;
            if constexpr (SIGN < 0) {
                cp_async16(b + pair_slot(p, l), src + ((long)z * N + p) * pp + prc, ok);
            } else {
                const int ci = band_compact_index(a.band, p);
                cp_async16(b + pair_slot(p, l), src + ((long)z * nb + (ci >= 0 ? ci : 0)) * pp + prc, ok && ci >= 0);
            }
        }
        cp_async_commit();
    };
    long it = blockIdx.x;
    if (it < items) stage(it, buf0);
    for (int k = 0; it < items; it += gridDim.x, k ^= 1) {
        float4* cur = k ? buf1 : buf0;
        float4* nxt = k ? buf0 : buf1;
        cp_async_wait_all();
        cpx<float> va[E], vb[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const float4 q = cur[pair_slot(t + TPL * m, l)];
            va[m] = mk(q.x, q.y);
            vb[m] = mk(q.z, q.w);
        }
        // every thread has its pair in registers and the previous transform is
        // done: cur becomes this transform's exchange buffer, nxt the next stage
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        SFor<0, CPlan<N, E>::NST>::run(
            [&](auto sc) { pstage<N, E, decltype(sc)::value, SIGN>(va, vb, t, l, cur, tw); });
        const int z = (int)(it / ntile);
        const int pr = (int)(it - (long)z * ntile) * NP + l;
        if (pr < npair) {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int p = t + TPL * m;
                const float4 q = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
                if constexpr (SIGN < 0) {
                    const int ci = band_compact_index(a.band, p);
                    if (ci >= 0) dst[((long)z * nb + ci) * pp + pr] = q;
                } else {
                    dst[((long)z * N + p) * pp + pr] = q;
                }
            }
        }
    }
}

// ----------------------------------------------------------------------------
// z stage, forward (+ optional round trip), on column pairs (FP32, variant
// V = 8).  The pair's y-stage columns are staged and transformed together as
// in ypass_pair_kernel; the spectral side (symbols, added term, reductions,
// spectrum stores; zfwd_spectral) runs once per column of the pair.
// ----------------------------------------------------------------------------
template <int N, int MINB>
__global__ void __launch_bounds__(PairShape<N>::THREADS, MINB)
    zfwd_pair_kernel(ZFwdArgs<float> a, const cpx<float>* __restrict__ twN) {
    using S = PairShape<N>;
    using C = float;
    constexpr int E = S::E, TPL = S::TPL, NP = S::NP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* buf0 = reinterpret_cast<float4*>(smem_raw);
    float4* buf1 = buf0 + S::TILE;
    cpx<float>* stw = reinterpret_cast<cpx<float>*>(buf1 + S::TILE);
    C* kt = reinterpret_cast<C*>(stw + N);
    TwStage<N, E, float>::fill(stw, twN);
    fill_k_table<N>(kt);
    __syncthreads();
    const int l = threadIdx.x % NP, t = threadIdx.x / NP;
    const TwStage<N, E, float> tw{stw};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int pp = (a.px ? a.px : nx) / 2;  // row pitch of the y-stage arrays in pairs
    const int npair = (nx + 1) / 2;
    const int ntile = (npair + NP - 1) / NP;
    const long items = (long)nb * ntile;
    const ZFwdOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;  // spectra
    const long yplane = (long)nb * pp;
    const float4* __restrict__ src = reinterpret_cast<const float4*>(op.in);
    float4* __restrict__ yout = reinterpret_cast<float4*>(op.ys_out);
    const SymD<C> dmain = make_symd<C>(op.sym, op.sym_ab, a.norm);  // the 1/N^3 folded in
    const SymD<C> dadd = make_symd<C>(op.add_sym, op.add_ab, op.add_coef);
    ZAcc acc;
    auto stage = [&](long it, float4* b) {
        const int cy = (int)(it / ntile);
        const int pr = (int)(it - (long)cy * ntile) * NP + l;
        const bool ok = pr < npair;
        const long ycol = (long)cy * pp + (ok ? pr : npair - 1);
#pragma unroll
        for (int m = 0; m < E; ++m) cp_async16(b + pair_slot(t + TPL * m, l), src + (t + TPL * m) * yplane + ycol, ok);
        cp_async_commit();
    };
    long it0 = blockIdx.x;
    if (it0 < items) stage(it0, buf0);
    int kbuf = 0;
    for (long it = it0; it < items; it += gridDim.x, kbuf ^= 1) {
        float4* cur = kbuf ? buf1 : buf0;
        float4* nxt = kbuf ? buf0 : buf1;
        cp_async_wait_all();
        cpx<float> va[E], vb[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const float4 q = cur[pair_slot(t + TPL * m, l)];
            va[m] = mk(q.x, q.y);
            vb[m] = mk(q.z, q.w);
        }
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        SFor<0, CPlan<N, E>::NST>::run(
            [&](auto sc) { pstage<N, E, decltype(sc)::value, -1>(va, vb, t, l, cur, tw); });
        const int cy = (int)(it / ntile);
        const int pr = (int)(it - (long)cy * ntile) * NP + l;
        const int fy = band_fft_index(a.band, cy);
        zfwd_spectral_pair<N, E, TPL>(op, dmain, dadd, kt, t, cut, nb, plane, nx, cy, pr, fy, va, vb, acc);
        if (yout) {  // uniform over the block
            SFor<0, CPlan<N, E>::NST>::run(
                [&](auto sc) { pstage<N, E, decltype(sc)::value, +1>(va, vb, t, l, cur, tw); });
            if (pr < npair) {
#pragma unroll
                for (int m = 0; m < E; ++m)
                    yout[(t + TPL * m) * yplane + (long)cy * pp + pr] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
            }
        }
    }
    zfwd_partials(op, acc, a.partials + (long)(blockIdx.y * gridDim.x + blockIdx.x) * MAX_RED);
}

// ----------------------------------------------------------------------------
// z stage, inverse, on column pairs (FP32, variant V = 8), one source and up
// to ZMULTI outputs per op as zinv_multi_c_kernel: the pair's two source
// columns are loaded once, each output applies its symbol to both, and the
// pair is transformed and stored as 16-byte vectors.
// ----------------------------------------------------------------------------
template <int N, int MINB>
__global__ void __launch_bounds__(PairShape<N>::THREADS, MINB)
    zinv_multi_pair_kernel(ZInvMultiArgs<float> a, const cpx<float>* __restrict__ twN) {
    using S = PairShape<N>;
    using C = float;
    constexpr int E = S::E, TPL = S::TPL, NP = S::NP, CH = E;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* xch = reinterpret_cast<float4*>(smem_raw);
    cpx<float>* stw = reinterpret_cast<cpx<float>*>(xch + S::TILE);
    C* kt = reinterpret_cast<C*>(stw + N);
    TwStage<N, E, float>::fill(stw, twN);
    fill_k_table<N>(kt);
    __syncthreads();
    const int l = threadIdx.x % NP, t = threadIdx.x / NP;
    const TwStage<N, E, float> tw{stw};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int pp = (a.px ? a.px : nx) / 2;  // row pitch of the y-stage arrays in pairs
    const int npair = (nx + 1) / 2;
    const int ntile = (npair + NP - 1) / NP;
    const long items = (long)nb * ntile;
    const ZInvMultiOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;  // spectra
    const long yplane = (long)nb * pp;
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const int cy = (int)(it / ntile);
        const int pr = (int)(it - (long)cy * ntile) * NP + l;
        const int fy = band_fft_index(a.band, cy);
        const C oy = kt[N + fy], ky2 = kt[fy] * kt[fy];
        const int kx0 = 2 * pr, kx1 = 2 * pr + 1;
        const bool ok0 = kx0 < nx, ok1 = kx1 < nx;
        const int col0 = cy * nx + (ok0 ? kx0 : nx - 1), col1 = cy * nx + (ok1 ? kx1 : nx - 1);
        const int kc0 = col0 - cy * nx, kc1 = col1 - cy * nx;
        const C ox0 = kt[N + kc0], ox1 = kt[N + kc1];
        const C kxy0 = kt[kc0] * kt[kc0] + ky2, kxy1 = kt[kc1] * kt[kc1] + ky2;
        const ZCol<N, TPL> idx0{t, cut, nb, plane, col0, ok0}, idx1{t, cut, nb, plane, col1, ok1};
        cpx<C> V0[E], V1[E];
        ld_chunk<CH>(op.spec, op.f64, idx0, 0, V0);
        ld_chunk<CH>(op.spec, op.f64, idx1, 0, V1);
#pragma unroll 1
        for (int o = 0; o < op.nout; ++o) {
            const SymD<C> d = make_symd<C>(op.sym[o], op.ab[o], op.coef[o]);
            cpx<float> va[E], vb[E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int fz = t + TPL * m;
                const C kz = kt[fz], oz = kt[N + fz];
                const C ksq0 = kxy0 + kz * kz, ksq1 = kxy1 + kz * kz;
                const C ri0 = d.inv ? rinv_of(ksq0) : C(0), ri1 = d.inv ? rinv_of(ksq1) : C(0);
                va[m] = idx0.valid(m) ? sym_apply(d, ox0, oy, oz, ksq0, ri0, V0[m]) : mk(C(0), C(0));
                vb[m] = idx1.valid(m) ? sym_apply(d, ox1, oy, oz, ksq1, ri1, V1[m]) : mk(C(0), C(0));
            }
            SFor<0, CPlan<N, E>::NST>::run(
                [&](auto sc) { pstage<N, E, decltype(sc)::value, +1>(va, vb, t, l, xch, tw); });
            if (pr < npair) {
                float4* __restrict__ dst = reinterpret_cast<float4*>(op.ys_out[o]);
#pragma unroll
                for (int m = 0; m < E; ++m)
                    dst[(t + TPL * m) * yplane + (long)cy * pp + pr] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Column-per-warp (CW) y/z passes, variants V = 5, 6 of YShape.  A block holds
// a tile of TX columns x N rows in shared memory (TileMap).  Global memory is
// read and written in the staging mapping (thread = column ls of row
// ts + 32 m, so a warp covers whole 64-128-byte rows); each warp then
// transforms one column held as 32 threads x N/32 elements, exchanging
// through its own padded row with __syncwarp only.  Two block barriers per
// item (four for a z round trip) instead of two per FFT stage.
// ----------------------------------------------------------------------------
template <int N, int V, typename T>
struct CWGeom {
    using S = YShape<N, T, V>;
    static_assert(S::CW && S::TPLY == 32 && S::YTHREADS / S::TX == 32, "CW shape: one warp per column");
    static constexpr int E = S::EY, TX = S::TX, SR = 32;
    using TM = TileMap<TX, T>;
    int lane, w, ls, ts;
    __device__ __forceinline__ CWGeom()
        : lane(threadIdx.x & 31), w(threadIdx.x >> 5), ls(threadIdx.x % TX), ts(threadIdx.x / TX) {}
    // the warp's column of a tile into / out of registers (position lane + 32 m)
    __device__ __forceinline__ void col_load(const cpx<T>* tile, cpx<T> (&v)[E]) const {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = tile[TM::at(lane + 32 * m, w)];
    }
    __device__ __forceinline__ void col_store(cpx<T>* tile, const cpx<T> (&v)[E]) const {
#pragma unroll
        for (int m = 0; m < E; ++m) tile[TM::at(lane + 32 * m, w)] = v[m];
    }
    // slot of staging element m (row ts + 32 m, column ls)
    __device__ __forceinline__ int slot(int m) const { return TM::at(ts + SR * m, ls); }
};

template <int N, int V, int SIGN, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    ypass_cw_kernel(YArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using G = CWGeom<N, V, T>;
    constexpr int E = G::E, TX = G::TX, SR = G::SR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* tile0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* tile1 = tile0 + N * TX;
    cpx<T>* xch = tile1 + N * TX;
    cpx<T>* stw = xch + TX * S::WPITCH;
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    __syncthreads();
    const G g;
    const TwTab<N, E, T> tw{stw};
    const RowMap<E> xmap{g.w * S::WPITCH};
    const int nx = a.nx, nb = a.band.nb;
    const int px = a.px ? a.px : nx;  // row pitch of xs and ys
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)a.nz * ntile;
    const cpx<T>* __restrict__ src = a.in[blockIdx.y];
    cpx<T>* __restrict__ dst = a.out[blockIdx.y];
    auto stage = [&](long it, cpx<T>* b) {
        const int z = (int)(it / ntile);
        const int kx = (int)(it - (long)z * ntile) * TX + g.ls;
        const bool ok = kx < nx;
        const int kxc = ok ? kx : nx - 1;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int p = g.ts + SR * m;
            if constexpr (SIGN < 0) {
                cp_async_elem(b + g.slot(m), src + ((long)z * N + p) * px + kxc, ok);
            } else {
                const int ci = band_compact_index(a.band, p);
                cp_async_elem(b + g.slot(m), src + ((long)z * nb + (ci >= 0 ? ci : 0)) * px + kxc, ok && ci >= 0);
            }
        }
        cp_async_commit();
    };
    long it = blockIdx.x;
    if (it < items) stage(it, tile0);
    for (int k = 0; it < items; it += gridDim.x, k ^= 1) {
        cpx<T>* cur = k ? tile1 : tile0;
        cpx<T>* nxt = k ? tile0 : tile1;
        cp_async_wait_all();
        // the tile is complete, and every thread is done storing the item
        // that last used nxt
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        cpx<T> v[E];
        g.col_load(cur, v);
        cfft<N, E, SIGN, SyncWarp>(v, g.lane, xch, xmap, tw);
        g.col_store(cur, v);
        __syncthreads();
        const int z = (int)(it / ntile);
        const int kx = (int)(it - (long)z * ntile) * TX + g.ls;
        if (kx < nx) {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int p = g.ts + SR * m;
                if constexpr (SIGN < 0) {
                    const int ci = band_compact_index(a.band, p);
                    if (ci >= 0) dst[((long)z * nb + ci) * px + kx] = cur[g.slot(m)];
                } else {
                    dst[((long)z * N + p) * px + kx] = cur[g.slot(m)];
                }
            }
        }
    }
}

template <int N, int V, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    zfwd_cw_kernel(ZFwdArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using G = CWGeom<N, V, T>;
    using C = T;
    constexpr int E = G::E, TX = G::TX, SR = G::SR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* tile0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* tile1 = tile0 + N * TX;
    cpx<T>* xch = tile1 + N * TX;
    cpx<T>* stw = xch + TX * S::WPITCH;
    C* kt = reinterpret_cast<C*>(stw + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    fill_k_table<N>(kt);
    __syncthreads();
    const G g;
    const TwTab<N, E, T> tw{stw};
    const RowMap<E> xmap{g.w * S::WPITCH};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)nb * ntile;
    const ZFwdOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;                      // spectra
    const int px = a.px ? a.px : nx, yplane = nb * px;  // y-stage arrays
    const cpx<T>* __restrict__ src = reinterpret_cast<const cpx<T>*>(op.in);
    cpx<T>* __restrict__ yout = reinterpret_cast<cpx<T>*>(op.ys_out);
    const SymD<C> dmain = make_symd<C>(op.sym, op.sym_ab, a.norm);  // the 1/N^3 folded in
    const SymD<C> dadd = make_symd<C>(op.add_sym, op.add_ab, op.add_coef);
    ZAcc acc;
    auto stage = [&](long it, cpx<T>* b) {
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + g.ls;
        const bool ok = kx < nx;
        const int ycol = cy * px + (ok ? kx : nx - 1);
#pragma unroll
        for (int m = 0; m < E; ++m) cp_async_elem(b + g.slot(m), src + (g.ts + SR * m) * yplane + ycol, ok);
        cp_async_commit();
    };
    long it0 = blockIdx.x;
    if (it0 < items) stage(it0, tile0);
    int kbuf = 0;
    for (long it = it0; it < items; it += gridDim.x, kbuf ^= 1) {
        cpx<T>* cur = kbuf ? tile1 : tile0;
        cpx<T>* nxt = kbuf ? tile0 : tile1;
        cp_async_wait_all();
        __syncthreads();
        if (it + gridDim.x < items) stage(it + gridDim.x, nxt);
        cpx<T> v[E];
        g.col_load(cur, v);
        cfft<N, E, -1, SyncWarp>(v, g.lane, xch, xmap, tw);
        g.col_store(cur, v);
        __syncthreads();
        // spectral side in the staging mapping (coalesced spectrum accesses)
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + g.ls;
        const bool ok = kx < nx;
        const int col = cy * nx + (ok ? kx : nx - 1);  // clamped: loads stay in bounds
        const ZCol<N, SR> idx{g.ts, cut, nb, plane, col, ok};
        cpx<C> Y[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const cpx<T> y = cur[g.slot(m)];
            Y[m] = mk((C)y.x, (C)y.y);
        }
        zfwd_spectral<N, E, SR>(op, dmain, dadd, kt, idx, band_fft_index(a.band, cy), col - cy * nx,
                                kx_weight(N, kx), Y, acc);
        if (yout) {  // uniform over the block
#pragma unroll
            for (int m = 0; m < E; ++m) cur[g.slot(m)] = mk((T)Y[m].x, (T)Y[m].y);
            __syncthreads();
            g.col_load(cur, v);
            cfft<N, E, +1, SyncWarp>(v, g.lane, xch, xmap, tw);
            g.col_store(cur, v);
            __syncthreads();
            if (ok) {
#pragma unroll
                for (int m = 0; m < E; ++m) yout[(g.ts + SR * m) * yplane + cy * px + kx] = cur[g.slot(m)];
            }
        }
    }
    zfwd_partials(op, acc, a.partials + (long)(blockIdx.y * gridDim.x + blockIdx.x) * MAX_RED);
}

template <int N, int V, typename T>
__global__ void __launch_bounds__(YShape<N, T, V>::YTHREADS, YShape<N, T, V>::YMINB)
    zinv_cw_kernel(ZInvArgs<T> a, const cpx<T>* __restrict__ twN) {
    using S = YShape<N, T, V>;
    using G = CWGeom<N, V, T>;
    using C = T;
    constexpr int E = G::E, TX = G::TX, SR = G::SR, CH = E < 8 ? E : 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* tile0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* tile1 = tile0 + N * TX;
    cpx<T>* xch = tile1 + N * TX;
    cpx<T>* stw = xch + TX * S::WPITCH;
    C* kt = reinterpret_cast<C*>(stw + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) stw[i] = twN[i];
    fill_k_table<N>(kt);
    __syncthreads();
    const G g;
    const TwTab<N, E, T> tw{stw};
    const RowMap<E> xmap{g.w * S::WPITCH};
    const int nx = a.nx, nb = a.band.nb, cut = a.band.cut;
    const int ntile = (nx + TX - 1) / TX;
    const long items = (long)nb * ntile;
    const ZInvOp& op = a.op[blockIdx.y];
    const int plane = nb * nx;                      // spectra
    const int px = a.px ? a.px : nx, yplane = nb * px;  // y-stage arrays
    const int nsrc = op.nsrc;
    cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(op.ys_out);
    int kbuf = 0;
    for (long it = blockIdx.x; it < items; it += gridDim.x, kbuf ^= 1) {
        // two tiles alternate, so this item's staging writes never meet the
        // previous item's stores (the barrier after them orders the one before)
        cpx<T>* cur = kbuf ? tile1 : tile0;
        const int cy = (int)(it / ntile);
        const int kx = (int)(it - (long)cy * ntile) * TX + g.ls;
        const bool ok = kx < nx;
        const int col = cy * nx + (ok ? kx : nx - 1);  // clamped: loads stay in bounds
        const int fy = band_fft_index(a.band, cy);
        const int kxc = col - cy * nx;
        const C ox = kt[N + kxc], oy = kt[N + fy];
        const C kxy2 = kt[kxc] * kt[kxc] + kt[fy] * kt[fy];
        const ZCol<N, SR> idx{g.ts, cut, nb, plane, col, ok};
        cpx<C> Y[E];
#pragma unroll
        for (int m = 0; m < E; ++m) Y[m] = mk(C(0), C(0));
#pragma unroll 1
        for (int s = 0; s < nsrc; ++s) {
            const void* spec = op.src[s].spec;
            const int f64 = op.src[s].f64;
            const SymD<C> d = make_symd<C>(op.src[s].sym, op.src[s].ab, op.src[s].coef);
#pragma unroll
            for (int m0 = 0; m0 < E; m0 += CH) {
                cpx<C> Vv[CH];
                ld_chunk<CH>(spec, f64, idx, m0, Vv);
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int fz = g.ts + SR * (m0 + j);
                    const C kz = kt[fz], oz = kt[N + fz];
                    const C ksq = kxy2 + kz * kz;
                    const C ri = d.inv ? rinv_of(ksq) : C(0);
                    if (idx.valid(m0 + j)) Y[m0 + j] = Y[m0 + j] + sym_apply(d, ox, oy, oz, ksq, ri, Vv[j]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < E; ++m) cur[g.slot(m)] = mk((T)Y[m].x, (T)Y[m].y);
        __syncthreads();
        cpx<T> v[E];
        g.col_load(cur, v);
        cfft<N, E, +1, SyncWarp>(v, g.lane, xch, xmap, tw);
        g.col_store(cur, v);
        __syncthreads();
        if (ok) {
#pragma unroll
            for (int m = 0; m < E; ++m) dst[(g.ts + SR * m) * yplane + cy * px + kx] = cur[g.slot(m)];
        }
    }
}

}  // namespace mlq
