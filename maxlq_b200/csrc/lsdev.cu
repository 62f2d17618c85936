// lsdev.cu -- the line search of maxdLqdt on the device: the controller and
// the bookkeeping kernels of the conditional graph that runs mnbrak and Brent
// (optimization.f90:613-951) without a host round trip per trial.
//
// Compiled without multiply-add contraction (-fmad=false) so that every
// trial value and every step of the search rounds as on the host.
#include "linesearch.cuh"

namespace mlq {

namespace {

__device__ bool ls_memo_add(LsDevState* s, double tau, const double R[3], double lqq, int fft) {
    const int k = s->ntr;
    if (k >= LS_MEMO) return false;
    s->mtau[k] = tau;
    for (int i = 0; i < 3; ++i) s->mR[k][i] = R[i];
    s->mlqq[k] = lqq;
    s->mfft[k] = fft;
    s->ntr = k + 1;
    return true;
}

// J(tau) from the table, or from the polynomials inside [tlo, thi];
// anything else suspends the search at tau.
struct DevEval {
    LsDevState* s;
    int count = 0;
    int err = 0;
    double ptau = 0.0;
    __device__ bool operator()(double tau, double* J) {
        ++count;
        const LsParams& p = s->par;
        int k = -1;
        for (int i = 0; i < s->ntr; ++i)
            if (s->mtau[i] == tau) {
                k = i;
                break;
            }
        if (k < 0) {
            if (p.transform_trials || !ls_free(s->poly, tau)) {
                ptau = tau;
                return false;
            }
            double R[3], lqq;
            ls_poly_R(s->poly, p.q, p.cv, p.cp, tau, R, &lqq);
            if (!ls_memo_add(s, tau, R, lqq, 0)) {
                err = LS_ERR_CAP;
                return false;
            }
            k = s->ntr - 1;
        }
        *J = ls_J(s->mR[k][1], s->mR[k][2], s->mlqq[k], p.q, p.B);
        if (isnan(*J)) {
            err = MLQ_ERR_NAN;
            return false;
        }
        return true;
    }
};

__device__ void ls_stop(LsDevState* s, int status, cudaGraphConditionalHandle h_loop,
                        cudaGraphConditionalHandle h_chk) {
    s->out.status = status;
    cudaGraphSetConditional(h_loop, 0);
    cudaGraphSetConditional(h_chk, 0);
}

}  // namespace

// The coefficients of this line search from the setup's sums (results[100..],
// [140..], [149..]) and the per-block interval ends (partials, 2 per block);
// clears the table for a new search.
__global__ void ls_coef_kernel(LsDevState* s, const double* __restrict__ results,
                               const double* __restrict__ partials, int nblocks, LsAnchorSet an) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    // one warp: each lane takes every 32nd block, then a shuffle tree (max and
    // min are exact, so any order gives the same ends)
    constexpr int K = LS_ANCHORS + 1, W = 2 * K;
    const int lane = threadIdx.x;
    double lo[K], hi[K];
    for (int k = 0; k < K; ++k) {
        lo[k] = -1e300;
        hi[k] = 1e300;
    }
    for (int g = lane; g < nblocks; g += 32)
        for (int k = 0; k < K; ++k) {
            lo[k] = fmax(lo[k], partials[W * g + 2 * k]);
            hi[k] = fmin(hi[k], partials[W * g + 2 * k + 1]);
        }
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmax(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmin(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    if (lane != 0) return;
    ls_assemble(results + 100, results + 140, results + 149, lo[0], hi[0], lo + 1, hi + 1, an.a, s->poly);
    s->ntr = 0;
    s->need = 0;
    s->ptau = 0.0;
    s->out = LsOut{};
    s->out.status = LS_RUNNING;
}

// One pass of the controller: mnbrak then Brent from the start over the
// table; ends the loop when the search completes (or fails), else leaves
// the first tau without a value in ptau and opens the check branch.
__global__ void ls_ctrl_kernel(LsDevState* s, cudaGraphConditionalHandle h_loop, cudaGraphConditionalHandle h_chk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    LsOut& o = s->out;
    if (o.status != LS_RUNNING) {
        ls_stop(s, o.status, h_loop, h_chk);
        return;
    }
    if (o.loops >= LS_MAX_LOOPS) {
        ls_stop(s, LS_ERR_CAP, h_loop, h_chk);
        return;
    }
    ++o.loops;
    DevEval ev{s};
    double tb[2] = {0.0, 0.0}, x = 0.0, fx = 0.0;
    int mflag = 0;
    int r = ls_mnbrak(ev, s->par.tA0, s->par.tB0, tb, &mflag);
    if (r == 0) r = ls_brent(ev, tb, &x, &fx);
    if (ev.err) {
        ls_stop(s, ev.err, h_loop, h_chk);
        return;
    }
    if (r == LS_SUSPEND) {
        s->need = 1;
        s->ptau = ev.ptau;
        ++o.checks;
        cudaGraphSetConditional(h_loop, 1);
        cudaGraphSetConditional(h_chk, 1);
        return;
    }
    o.mflag = mflag;
    o.tb[0] = tb[0];
    o.tb[1] = tb[1];
    o.evals = ev.count;
    for (int i = 0; i < s->ntr; ++i) {
        if (s->mfft[i])
            ++o.nfft;
        else
            ++o.npoly;
    }
    if (mflag == 0) {
        o.tau1 = x;
        o.fx = fx;
        for (int i = 0; i < s->ntr; ++i)
            if (s->mtau[i] == x) {
                for (int c = 0; c < 3; ++c) o.R1[c] = s->mR[i][c];
                o.lqq1 = s->mlqq[i];
                o.fft1 = s->mfft[i];
                break;
            }
    }
    ls_stop(s, 0, h_loop, h_chk);
}

// After the minimum of S(ptau) over the points (per-block minima in
// partials): the polynomial value where S >= 0 everywhere, else open the
// transform branch.
__global__ void ls_check_kernel(LsDevState* s, const double* __restrict__ partials, int nblocks,
                                cudaGraphConditionalHandle h_fft) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mn = 1e300;
    for (int g = 0; g < nblocks; ++g) mn = fmin(mn, partials[g]);
    if (mn >= 0.0 && !s->par.transform_trials) {
        double R[3], lqq;
        ls_poly_R(s->poly, s->par.q, s->par.cv, s->par.cp, s->ptau, R, &lqq);
        if (!ls_memo_add(s, s->ptau, R, lqq, 0)) s->out.status = LS_ERR_CAP;
        s->need = 0;
        cudaGraphSetConditional(h_fft, 0);
    } else {
        s->need = 2;
        cudaGraphSetConditional(h_fft, 1);
    }
}

// After the transform trial at ptau: its sums r[0..3] give the value.
__global__ void ls_fft_kernel(LsDevState* s, const double* __restrict__ r) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double R[3], lqq;
    ls_fft_R(s->poly, s->par.q, s->par.cv, s->par.cp, r, s->ptau, R, &lqq);
    if (!ls_memo_add(s, s->ptau, R, lqq, 1)) s->out.status = LS_ERR_CAP;
    s->need = 0;
}

void ls_launch_coef(LsDevState* s, const double* results, const double* partials, int nblocks, const LsAnchorSet& an,
                    cudaStream_t st) {
    ls_coef_kernel<<<1, 32, 0, st>>>(s, results, partials, nblocks, an);
}
void ls_launch_ctrl(LsDevState* s, cudaGraphConditionalHandle h_loop, cudaGraphConditionalHandle h_chk,
                    cudaStream_t st) {
    ls_ctrl_kernel<<<1, 32, 0, st>>>(s, h_loop, h_chk);
}
void ls_launch_check(LsDevState* s, const double* partials, int nblocks, cudaGraphConditionalHandle h_fft,
                     cudaStream_t st) {
    ls_check_kernel<<<1, 32, 0, st>>>(s, partials, nblocks, h_fft);
}
void ls_launch_fft(LsDevState* s, const double* r, cudaStream_t st) { ls_fft_kernel<<<1, 32, 0, st>>>(s, r); }

}  // namespace mlq
