// regfft.cuh -- register-resident batched FFTs and the pass kernels built on them.
//
// A line of length L (a power of two) is owned by T = L/E threads; before and
// after every stage thread t holds the elements at positions t + T*m,
// m = 0..E-1, in registers.  A stage of radix R (R divides E) is E/R
// butterflies per thread in registers (Stockham autosort); between stages the
// outputs go through shared memory once (write, sync, read, sync).  The last
// stage leaves the natural-order result in the same register slots, so global
// loads and stores touch positions t + T*m: consecutive threads, consecutive
// addresses.  Lines are either the columns of a tile (y and z passes: lanes
// walk the contiguous kx axis) or contiguous rows (x passes).
#pragma once

#include "functors.cuh"
#include "kernels.cuh"

namespace mlq {

struct RPlan {
    int L;      // length (power of two)
    int nst;    // stages
    int radix[8];
    int tw_off; // offset of W_L in the twiddle pool (T precision)
};

template <int SIGN, typename T>
__device__ __forceinline__ cpx<T> twid(const cpx<T>* __restrict__ tw, int e) {
    const cpx<T> w = tw[e];
    return SIGN < 0 ? w : conj(w);
}

// one stage: E/R butterflies per thread
template <int R, int E, int SIGN, typename T, class SIdx>
__device__ __forceinline__ void reg_stage(cpx<T> (&v)[E], int t, int nT, int ns, int lg_ns, int L, bool last,
                                          cpx<T>* sm, const SIdx& si, const cpx<T>* __restrict__ tw) {
    constexpr int Q = E / R;
    const int step = L / (ns * R);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int b = t + nT * i;
        const int k = b & (ns - 1);
        cpx<T> a[R];
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = v[i + Q * r];
        if (ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) a[r] = a[r] * twid<SIGN>(tw, r * k * step);
        }
        dftR<R, SIGN>(a);
        if (last) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[i + Q * r] = a[r];
        } else {
            const int base = ((b >> lg_ns) << lg_ns) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm[si(base + r * ns)] = a[r];
        }
    }
}

// Full transform of the thread's E register elements.  Must be called by
// every thread of the block (it synchronises); sm must not be in use.
template <int E, int SIGN, typename T, class SIdx>
__device__ __forceinline__ void reg_fft(cpx<T> (&v)[E], int t, int nT, const RPlan& pl, cpx<T>* sm, const SIdx& si,
                                        const cpx<T>* __restrict__ tw_pool) {
    const cpx<T>* tw = tw_pool + pl.tw_off;
    int ns = 1, lg = 0;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s];
        const bool last = s == pl.nst - 1;
        switch (R) {
            case 2: reg_stage<2, E, SIGN>(v, t, nT, ns, lg, pl.L, last, sm, si, tw); break;
            case 4: reg_stage<4, E, SIGN>(v, t, nT, ns, lg, pl.L, last, sm, si, tw); break;
            case 8: reg_stage<8, E, SIGN>(v, t, nT, ns, lg, pl.L, last, sm, si, tw); break;
            default:
                if constexpr (E % 16 == 0) reg_stage<16, E, SIGN>(v, t, nT, ns, lg, pl.L, last, sm, si, tw);
                break;
        }
        if (!last) {
            __syncthreads();
#pragma unroll
            for (int m = 0; m < E; ++m) v[m] = sm[si(t + nT * m)];
            __syncthreads();
        }
        ns *= R;
        lg += (R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4);
    }
}

// shared-memory index maps
struct ColIdx {  // tile columns: element p of column l at p*tx + l
    int tx, l;
    __device__ __forceinline__ int operator()(int p) const { return p * tx + l; }
};
struct RowIdx {  // contiguous rows, one pad element every 16
    int base;
    __device__ __forceinline__ int operator()(int p) const { return base + p + (p >> 4); }
};
__host__ __device__ __forceinline__ int row_pitch(int L) { return L + L / 16 + 1; }

// ----------------------------------------------------------------------------
// y pass.  grid = (ceil(nx/tx), n, narr), block = tx * (n/E)
// ----------------------------------------------------------------------------
template <int E, int SIGN, typename T>
__global__ void __launch_bounds__(256, 3) ypass_reg_kernel(YArgs<T> a, RPlan pl, const cpx<T>* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb, nT = n / E;
    const int l = threadIdx.x % tx, t = threadIdx.x / tx;
    const int kx = blockIdx.x * tx + l;
    const bool ok = kx < nx;
    const int z = blockIdx.y;
    const cpx<T>* __restrict__ src = a.in[blockIdx.z];
    cpx<T>* __restrict__ dst = a.out[blockIdx.z];
    cpx<T> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int p = t + nT * m;
        if (SIGN < 0) {
            v[m] = ok ? src[((long)z * n + p) * nx + kx] : czero<T>();
        } else {
            const int ci = band_compact_index(a.band, p);
            v[m] = (ok && ci >= 0) ? src[((long)z * nb + ci) * nx + kx] : czero<T>();
        }
    }
    reg_fft<E, SIGN>(v, t, nT, pl, sm, ColIdx{tx, l}, tw);
    if (!ok) return;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int p = t + nT * m;
        if (SIGN < 0) {
            const int ci = band_compact_index(a.band, p);
            if (ci >= 0) dst[((long)z * nb + ci) * nx + kx] = v[m];
        } else {
            dst[((long)z * n + p) * nx + kx] = v[m];
        }
    }
}

// ----------------------------------------------------------------------------
// z stage, forward (+ optional round trip).  grid = (ceil(nx/tx), nb, narr)
// ----------------------------------------------------------------------------
template <int E, typename T>
__global__ void __launch_bounds__(256, 3) zfwd_reg_kernel(ZFwdArgs<T> a, RPlan pl, const cpx<T>* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb, nT = n / E;
    const int l = threadIdx.x % tx, t = threadIdx.x / tx;
    const int kx = blockIdx.x * tx + l;
    const bool ok = kx < nx;
    const int cy = blockIdx.y;
    const ZFwdOp& op = a.op[blockIdx.z];
    const long plane = (long)nb * nx;
    const cpx<T>* __restrict__ src = reinterpret_cast<const cpx<T>*>(op.in);
    cpx<T> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int p = t + nT * m;
        v[m] = ok ? src[(long)p * plane + (long)cy * nx + kx] : czero<T>();
    }
    const ColIdx si{tx, l};
    reg_fft<E, -1>(v, t, nT, pl, sm, si, tw);
    double acc_self = 0.0, acc_w0 = 0.0, acc_w1 = 0.0, acc_w2 = 0.0;
    const int fy = band_fft_index(a.band, cy);
    const double wgt = kx_weight(n, kx);
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int fz = t + nT * m;
        const int cz = band_compact_index(a.band, fz);
        cpx<double> Y = mk(0.0, 0.0);
        if (cz >= 0 && ok) {
            const Kvec k = make_k(n, kx, fy, fz);
            Y = apply_sym(op.sym, op.sym_ab, k, mk((double)v[m].x, (double)v[m].y) * a.norm);
            const long si2 = ((long)cz * nb + cy) * nx + kx;
            if (op.add) Y = Y + apply_sym(op.add_sym, op.add_ab, k, ld_spec(op.add, op.add_f64, si2)) * op.add_coef;
            if (op.red_self >= 0) acc_self += wgt * (Y.x * Y.x + Y.y * Y.y);
            if (op.red_with[0]) {
                const cpx<double> W = ld_spec(op.red_with[0], op.red_with_f64[0], si2);
                acc_w0 += wgt * (Y.x * W.x + Y.y * W.y);
            }
            if (op.red_with[1]) {
                const cpx<double> W = ld_spec(op.red_with[1], op.red_with_f64[1], si2);
                acc_w1 += wgt * (Y.x * W.x + Y.y * W.y);
            }
            if (op.red_with[2]) {
                const cpx<double> W = ld_spec(op.red_with[2], op.red_with_f64[2], si2);
                acc_w2 += wgt * (Y.x * W.x + Y.y * W.y);
            }
            if (op.spec_out) st_spec(op.spec_out, op.spec_f64, si2, Y);
        }
        v[m] = mk((T)Y.x, (T)Y.y);
    }
    const int block_lin = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    if (op.red_self >= 0 || op.red_with[0] || op.red_with[1] || op.red_with[2]) {
        double acc4[4] = {acc_self, acc_w0, acc_w1, acc_w2};
        __shared__ double part4[4];
        block_reduce_store<4>(acc4, part4, 0);
        __syncthreads();
        if (threadIdx.x < MAX_RED) {
            double v2 = 0.0;
            if ((int)threadIdx.x == op.red_self) v2 += part4[0];
            for (int r = 0; r < 3; ++r)
                if (op.red_with[r] && (int)threadIdx.x == op.red_with_slot[r]) v2 += part4[1 + r];
            a.partials[(long)block_lin * MAX_RED + threadIdx.x] = v2;
        }
    } else if (threadIdx.x < MAX_RED) {
        a.partials[(long)block_lin * MAX_RED + threadIdx.x] = 0.0;
    }
    if (!op.ys_out) return;
    reg_fft<E, +1>(v, t, nT, pl, sm, si, tw);
    if (!ok) return;
    cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(op.ys_out);
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int p = t + nT * m;
        dst[(long)p * plane + (long)cy * nx + kx] = v[m];
    }
}

// ----------------------------------------------------------------------------
// z stage, inverse from spectra.  grid = (ceil(nx/tx), nb, narr)
// ----------------------------------------------------------------------------
template <int E, typename T>
__global__ void __launch_bounds__(256, 3) zinv_reg_kernel(ZInvArgs<T> a, RPlan pl, const cpx<T>* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    const int n = a.n, tx = a.tx, nx = a.nx, nb = a.band.nb, nT = n / E;
    const int l = threadIdx.x % tx, t = threadIdx.x / tx;
    const int kx = blockIdx.x * tx + l;
    const bool ok = kx < nx;
    const int cy = blockIdx.y;
    const ZInvOp& op = a.op[blockIdx.z];
    const int fy = band_fft_index(a.band, cy);
    cpx<T> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int fz = t + nT * m;
        const int cz = band_compact_index(a.band, fz);
        cpx<double> Y = mk(0.0, 0.0);
        if (cz >= 0 && ok) {
            const Kvec k = make_k(n, kx, fy, fz);
            const long si2 = ((long)cz * nb + cy) * nx + kx;
            for (int s = 0; s < op.nsrc; ++s)
                Y = Y + apply_sym(op.src[s].sym, op.src[s].ab, k, ld_spec(op.src[s].spec, op.src[s].f64, si2)) *
                            op.src[s].coef;
        }
        v[m] = mk((T)Y.x, (T)Y.y);
    }
    reg_fft<E, +1>(v, t, nT, pl, sm, ColIdx{tx, l}, tw);
    if (!ok) return;
    cpx<T>* __restrict__ dst = reinterpret_cast<cpx<T>*>(op.ys_out);
    const long plane = (long)nb * nx;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int p = t + nT * m;
        dst[(long)p * plane + (long)cy * nx + kx] = v[m];
    }
}

// ----------------------------------------------------------------------------
// x stage, forward: functor + real FFT along x.  Each CTA owns lx rows; the
// NOUT*lx output rows are transformed as complex rows of length h = n/2 (pairs
// of reals), T = h/E threads per row.  block = NOUT * lx * T threads.
// ----------------------------------------------------------------------------
template <int E, typename T, class F>
__global__ void __launch_bounds__(256, 3) xfwd_reg_kernel(XFwdArgs<T> a, F f, RPlan pl, const cpx<T>* __restrict__ tw) {
    constexpr int NIN = F::NIN, NOUT = F::NOUT, NR = F::NRED;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    const int n = a.n, h = n / 2, lx = a.lx, nT = h / E;
    const int LP = row_pitch(h);
    const long line0 = (long)blockIdx.x * lx;
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    // 1. functor on pairs of points (2p, 2p+1); packed complex rows in smem
    for (int q = threadIdx.x; q < lx * h; q += blockDim.x) {
        const int l = q / h, p = q - l * h;
        const long g = (line0 + l) * n + 2 * p;
        T in0[NIN], in1[NIN];
#pragma unroll
        for (int i = 0; i < NIN; ++i) {
            const cpx<T> two = *reinterpret_cast<const cpx<T>*>(a.in[i] + g);
            in0[i] = two.x;
            in1[i] = two.y;
        }
        T o0[NOUT > 0 ? NOUT : 1], o1[NOUT > 0 ? NOUT : 1];
        f(in0, o0, acc);
        f(in1, o1, acc);
#pragma unroll
        for (int o = 0; o < NOUT; ++o) sm[(o * lx + l) * LP + p + (p >> 4)] = mk(o0[o], o1[o]);
    }
    __syncthreads();
    // 2. complex FFT of every packed row
    const int row = threadIdx.x / nT, t = threadIdx.x - row * nT;
    const RowIdx si{row * LP};
    cpx<T> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[si(t + nT * m)];
    __syncthreads();
    reg_fft<E, -1>(v, t, nT, pl, sm, si, tw);
    if (a.nanflag && t == 0 && !cpx_finite(v[0])) *a.nanflag = 1.0;  // the DC bin of the row
#pragma unroll
    for (int m = 0; m < E; ++m) sm[si(t + nT * m)] = v[m];
    __syncthreads();
    // 3. half spectrum of the real rows: X[k] = E[k] + W_n^k O[k], k < nx
    const cpx<T>* __restrict__ twn = tw + a.tw_n_off;
    for (int q = threadIdx.x; q < NOUT * lx * a.nx; q += blockDim.x) {
        const int r = q / a.nx, k = q - r * a.nx;
        const int o = r / lx, l = r - o * lx;
        const int base = r * LP;
        const int i1 = k & (h - 1), i2 = (h - k) & (h - 1);
        const cpx<T> zk = sm[base + i1 + (i1 >> 4)];
        const cpx<T> zc = conj(sm[base + i2 + (i2 >> 4)]);
        const cpx<T> Ev = (zk + zc) * T(0.5);
        const cpx<T> D = (zk - zc) * T(0.5);
        const cpx<T> O = mk<T>(D.y, -D.x);
        a.out[o][(line0 + l) * a.nx + k] = Ev + O * twn[k];
    }
    if constexpr (NR > 0) block_reduce_store<NR>(acc, a.partials, blockIdx.x);
}

// ----------------------------------------------------------------------------
// x stage, inverse (c2r).  grid = (n*n/lx, narr), block = lx * T, T = h/E.
// ----------------------------------------------------------------------------
template <int E, typename T>
__global__ void __launch_bounds__(256, 3) xinv_reg_kernel(XInvArgs<T> a, RPlan pl, const cpx<T>* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* sm = reinterpret_cast<cpx<T>*>(smem_raw);
    const int n = a.n, h = n / 2, lx = a.lx, nT = h / E;
    const int LP = row_pitch(h + 1);
    const long line0 = (long)blockIdx.x * lx;
    const cpx<T>* __restrict__ src = a.in[blockIdx.y];
    // 1. the half spectra (kx < nx_in, zero above), Hermitian part on kx = 0, h
    for (int q = threadIdx.x; q < lx * (h + 1); q += blockDim.x) {
        const int l = q / (h + 1), k = q - l * (h + 1);
        cpx<T> x = k < a.nx_in ? src[(line0 + l) * a.nx_in + k] : czero<T>();
        if (k == 0 || k == h) x.y = T(0);
        sm[l * LP + k + (k >> 4)] = x;
    }
    __syncthreads();
    const int row = threadIdx.x / nT, t = threadIdx.x - row * nT;
    const cpx<T>* __restrict__ twn = tw + a.tw_n_off;
    cpx<T> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int k = t + nT * m, kc = h - k;
        const cpx<T> xk = sm[row * LP + k + (k >> 4)];
        const cpx<T> xc = conj(sm[row * LP + kc + (kc >> 4)]);
        const cpx<T> Fk = xk + xc;
        const cpx<T> G = (xk - xc) * conj(twn[k]);
        v[m] = Fk + mk<T>(-G.y, G.x);
    }
    __syncthreads();
    const RowIdx si{row * LP};
    reg_fft<E, +1>(v, t, nT, pl, sm, si, tw);
    T* __restrict__ dst = a.out[blockIdx.y] + (line0 + row) * n;
#pragma unroll
    for (int m = 0; m < E; ++m) reinterpret_cast<cpx<T>*>(dst)[t + nT * m] = v[m];
}

}  // namespace mlq
