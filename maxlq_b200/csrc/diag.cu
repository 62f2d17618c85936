// diag.cu -- diagnostics of the state spectra: the shell energy spectrum and
// the enstrophy (maxdLpdt.f90:263-299, optimization.f90:119-123, 377-384).
//
// Both are sums over the pruned half spectrum of a band-limited field (every
// CG vector): by Parseval the reference's physical-space and full-spectrum
// sums are these sums with weight 2 for kx > 0 (the conjugate half).
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace mlq {

static const double PI_DIAG = 4.0 * std::atan2(1.0, 1.0);  // initialize.f90:164

// One block per shell: the energies sum_c |u_c|^2 of the shell's modes, in
// the fixed order of its mode list, times scale.
template <typename V>
__global__ void __launch_bounds__(256) shell_energy_kernel(SpecGeom g, const V* __restrict__ u,
                                                           const int* __restrict__ modes,
                                                           const int* __restrict__ off, double scale,
                                                           double* __restrict__ out) {
    const int sh = blockIdx.x;
    double s = 0.0;
    for (int k = off[sh] + threadIdx.x; k < off[sh + 1]; k += blockDim.x) {
        const int m = modes[k];
        const int fx = m % g.nx;
        double e = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double2 v = ldv(u, (long)c * g.ncomp + m);
            e += v.x * v.x + v.y * v.y;
        }
        s += kx_weight(g.n, fx) * e;
    }
    __shared__ double red[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        out[sh] = t * scale;
    }
}

void EngineBase::spectrum(const SVec* u, bool normalize, double* out) {
    const SpecGeom g = geom(b2);
    if (!d_shell_modes_) {
        // shell i of each mode: 2 pi i < |K| <= 2 pi (i + 1) with |K| and the
        // bounds formed as the reference forms them (function_ops.f90:2641-2652)
        std::vector<std::vector<int>> lists(n);
        auto sj = [&](int ci) { return ci <= b2.cut ? ci : ci - b2.nb; };
        for (int cz = 0; cz < b2.nb; ++cz)
            for (int cy = 0; cy < b2.nb; ++cy)
                for (int fx = 0; fx < b2.nx; ++fx) {
                    const double K1 = 2.0 * PI_DIAG * (double)fx, K2 = 2.0 * PI_DIAG * (double)sj(cy),
                                 K3 = 2.0 * PI_DIAG * (double)sj(cz);
                    const double nk = std::sqrt(K1 * K1 + K2 * K2 + K3 * K3);
                    const int i0 = (int)std::floor(nk / (2.0 * PI_DIAG));
                    for (int i = std::max(0, i0 - 1); i <= i0 + 1 && i < n; ++i) {
                        const double kk_min = 2.0 * PI_DIAG * (double)i, kk_max = 2.0 * PI_DIAG * (double)(i + 1);
                        if (kk_min < nk && nk <= kk_max) {
                            lists[i].push_back((int)(((long)cz * b2.nb + cy) * b2.nx + fx));
                            break;
                        }
                    }
                }
        std::vector<int> off(n + 1, 0), modes;
        modes.reserve((size_t)g.ncomp);
        for (int i = 0; i < n; ++i) {
            modes.insert(modes.end(), lists[i].begin(), lists[i].end());
            off[i + 1] = (int)modes.size();
        }
        d_shell_modes_ = (int*)dev_alloc(std::max<size_t>(modes.size(), 1) * sizeof(int));
        d_shell_off_ = (int*)dev_alloc(off.size() * sizeof(int));
        MLQ_CUDA(cudaMemcpyAsync(d_shell_modes_, modes.data(), modes.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 stream));
        MLQ_CUDA(cudaMemcpyAsync(d_shell_off_, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));  // the host vectors go out of scope
    }
    ensure_partials(n);
    // fftfwd is unnormalised: |N^3 u_hat|^2
    const double scale = (double)n3 * (double)n3;
    cudaEvent_t ev = prof_mark();
    if (state32_)
        shell_energy_kernel<float2><<<n, 256, 0, stream>>>(g, (const float2*)u, d_shell_modes_, d_shell_off_, scale,
                                                          d_partials);
    else
        shell_energy_kernel<double2><<<n, 256, 0, stream>>>(g, (const double2*)u, d_shell_modes_, d_shell_off_, scale,
                                                           d_partials);
    launched("spec_shells", 3.0 * sv_elem() * g.ncomp, ev);
    std::vector<double> sh(n);
    MLQ_CUDA(cudaMemcpyAsync(sh.data(), d_partials, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    for (int i = 0; i < n; ++i) {
        out[i] = 2.0 * PI_DIAG * (double)(i + 1);
        out[n + i] = sh[i];
    }
    if (normalize) {  // normalizeSpectrumByL2Norm (global_variables.f90:76; function_ops.f90:2666-2670)
        const SpecDotPair p = {u, u, 0};
        double l2 = 0.0;
        dots(&p, 1, &l2);
        double tot = 0.0;
        for (int i = 0; i < n; ++i) tot += out[n + i];
        const double spectral_Ener = 2.0 * PI_DIAG * tot;
        for (int i = 0; i < n; ++i) out[n + i] = l2 / spectral_Ener * out[n + i];
    }
}

double EngineBase::enstrophy(const SVec* u) {
    const SpecDotPair p = {u, nullptr, 3};
    double w2 = 0.0;
    dots(&p, 1, &w2);
    return 0.5 * w2;
}

}  // namespace mlq
