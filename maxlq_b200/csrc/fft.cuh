// fft.cuh -- shared-memory Stockham FFT for batches of short lines.
//
// A CTA holds `nl` lines of length L in shared memory, element (line l,
// index i) at buf[i*ls + l]: consecutive threads own consecutive lines, so
// every stage reads and writes bank-conflict-free.  Each stage is one radix-R
// butterfly per thread in registers (R in {2,3,4,8,16}), autosorting
// (Stockham) between two buffers, one __syncthreads per stage.  Twiddles come
// from a per-length FP64-accurate table W_L[k] = exp(-2 pi i k / L) built on
// the host.
#pragma once

#include "common.cuh"

namespace mlq {

constexpr int FFT_MAX_STAGES = 12;

struct FftPlan {
    int L;                       // transform length
    int nst;                     // number of stages
    int radix[FFT_MAX_STAGES];   // radix of each stage
    int tw_off;                  // offset of W_L in the twiddle pool
};

// --- radix-R DFT in registers ------------------------------------------------
// sqrt(1/2), cos(pi/8), sin(pi/8): mathematical constants.
#define MLQ_R2 0.70710678118654752440
#define MLQ_C8 0.92387953251128675613
#define MLQ_S8 0.38268343236508977173
#define MLQ_S3 0.86602540378443864676

template <int SIGN, typename T>
__device__ __forceinline__ void dft2(cpx<T>* v) {
    cpx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}

template <int SIGN, typename T>
__device__ __forceinline__ void dft3(cpx<T>* v) {
    cpx<T> t = v[1] + v[2];
    cpx<T> s = v[1] - v[2];
    cpx<T> m = v[0] - t * T(0.5);
    v[0] = v[0] + t;
    // SIGN<0: X1 = m - i*s3*s ; SIGN>0: X1 = m + i*s3*s
    cpx<T> r = rot90<SIGN>(s) * T(MLQ_S3);
    v[1] = m + r;
    v[2] = m - r;
}

template <int SIGN, typename T>
__device__ __forceinline__ void dft4(cpx<T>& a0, cpx<T>& a1, cpx<T>& a2, cpx<T>& a3) {
    cpx<T> t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = rot90<SIGN>(a1 - a3);
    a0 = t0 + t2;
    a2 = t0 - t2;
    a1 = t1 + t3;
    a3 = t1 - t3;
}

template <int SIGN, typename T>
__device__ __forceinline__ void dft4v(cpx<T>* v) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
}

template <int SIGN, typename T>
__device__ __forceinline__ cpx<T> w8(cpx<T> a, int k) {
    // a * exp(SIGN * 2 pi i k / 8), k in {1,2,3}
    const T r = T(MLQ_R2);
    if (k == 1) return mk<T>((a.x - SIGN * a.y) * r, (a.y + SIGN * a.x) * r);
    if (k == 2) return rot90<SIGN>(a);
    return mk<T>((-a.x - SIGN * a.y) * r, (-a.y + SIGN * a.x) * r);
}

template <int SIGN, typename T>
__device__ __forceinline__ void dft8(cpx<T>* v) {
    cpx<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cpx<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<SIGN>(e0, e1, e2, e3);
    dft4<SIGN>(o0, o1, o2, o3);
    o1 = w8<SIGN>(o1, 1);
    o2 = w8<SIGN>(o2, 2);
    o3 = w8<SIGN>(o3, 3);
    v[0] = e0 + o0;
    v[4] = e0 - o0;
    v[1] = e1 + o1;
    v[5] = e1 - o1;
    v[2] = e2 + o2;
    v[6] = e2 - o2;
    v[3] = e3 + o3;
    v[7] = e3 - o3;
}

template <int SIGN, typename T>
__device__ __forceinline__ void dft16(cpx<T>* v) {
    cpx<T> e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = v[2 * i];
        o[i] = v[2 * i + 1];
    }
    dft8<SIGN>(e);
    dft8<SIGN>(o);
    // twiddles exp(SIGN * 2 pi i k / 16), k = 0..7
    const T c1 = T(MLQ_C8), s1 = T(MLQ_S8), r2 = T(MLQ_R2);
    const T cs[8] = {T(1), c1, r2, s1, T(0), -s1, -r2, -c1};
    const T sn[8] = {T(0), s1, r2, c1, T(1), c1, r2, s1};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        cpx<T> w = mk<T>(cs[k], T(SIGN) * sn[k]);
        cpx<T> t = k == 0 ? o[k] : o[k] * w;
        v[k] = e[k] + t;
        v[k + 8] = e[k] - t;
    }
}

template <int R, int SIGN, typename T>
__device__ __forceinline__ void dftR(cpx<T>* v) {
    if (R == 2) dft2<SIGN>(v);
    if (R == 3) dft3<SIGN>(v);
    if (R == 4) dft4v<SIGN>(v);
    if (R == 8) dft8<SIGN>(v);
    if (R == 16) dft16<SIGN>(v);
}

// One Stockham stage of radix R over all lines.
template <int R, int SIGN, typename T>
__device__ __forceinline__ void stockham_stage(const cpx<T>* __restrict__ src, cpx<T>* __restrict__ dst, int L,
                                               int nl, int ls, int ns, const cpx<double>* __restrict__ tw,
                                               int tid, int nthr) {
    const int nb = L / R;
    const int total = nb * nl;
    const int step = L / (ns * R);
    for (int t = tid; t < total; t += nthr) {
        const int l = t % nl;
        const int j = t / nl;
        const int k = j % ns;
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            v[r] = src[(j + r * nb) * ls + l];
            if (r > 0 && k > 0) {
                const double2 wd = __ldg(reinterpret_cast<const double2*>(tw) + r * k * step);
                cpx<T> wt = mk<T>((T)wd.x, (T)(SIGN < 0 ? wd.y : -wd.y));
                v[r] = v[r] * wt;
            }
        }
        dftR<R, SIGN>(v);
        const int d = (j / ns) * ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(d + r * ns) * ls + l] = v[r];
    }
}

// Full transform; a holds the input, b is scratch of the same shape.  Returns
// the buffer holding the result.  Ends with a __syncthreads.
template <int SIGN, typename T>
__device__ cpx<T>* fft_lines(cpx<T>* a, cpx<T>* b, const FftPlan& pl, int nl, int ls, const cpx<double>* tw_pool,
                             int tid, int nthr) {
    const cpx<double>* tw = tw_pool + pl.tw_off;
    int ns = 1;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s];
        switch (R) {
            case 2: stockham_stage<2, SIGN>(a, b, pl.L, nl, ls, ns, tw, tid, nthr); break;
            case 3: stockham_stage<3, SIGN>(a, b, pl.L, nl, ls, ns, tw, tid, nthr); break;
            case 4: stockham_stage<4, SIGN>(a, b, pl.L, nl, ls, ns, tw, tid, nthr); break;
            case 8: stockham_stage<8, SIGN>(a, b, pl.L, nl, ls, ns, tw, tid, nthr); break;
            default: stockham_stage<16, SIGN>(a, b, pl.L, nl, ls, ns, tw, tid, nthr); break;
        }
        __syncthreads();
        cpx<T>* t = a;
        a = b;
        b = t;
        ns *= R;
    }
    return a;
}

}  // namespace mlq
