// common.cuh -- shared types for the maxLq B200 engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/maxlq.h"

namespace mlq {

// ----------------------------------------------------------------------------
// Complex arithmetic on float2 / double2 storage.
// ----------------------------------------------------------------------------
template <typename T>
struct cpx {
    T x, y;
};
template <>
struct __align__(8) cpx<float> {
    float x, y;
};
template <>
struct __align__(16) cpx<double> {
    double x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cpx<T> mk(T a, T b) {
    cpx<T> r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator*(cpx<T> a, T s) { return mk(a.x * s, a.y * s); }
template <typename T>
__host__ __device__ __forceinline__ cpx<T> conj(cpx<T> a) { return mk(a.x, -a.y); }
// multiply by -i (sign < 0) or +i (sign > 0)
template <int SIGN, typename T>
__host__ __device__ __forceinline__ cpx<T> rot90(cpx<T> a) {
    return SIGN < 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> czero() { return mk(T(0), T(0)); }

template <typename TO, typename TI>
__host__ __device__ __forceinline__ cpx<TO> ccast(cpx<TI> a) { return mk((TO)a.x, (TO)a.y); }

// ----------------------------------------------------------------------------
// A spectral band: the modes kept by a dealiasing cube cut.  cut = largest
// |j| kept on every axis; full = no cut (cut >= N/2).  Arrays in a band are
// stored "pruned": kx in [0, nx), ky/kz compact index in [0, nb) ordered
// 0..cut, -cut..-1 (or natural FFT order when full).
// ----------------------------------------------------------------------------
struct Band {
    int n;     // grid size
    int cut;   // largest |j| kept
    int nx;    // kx extent (cut+1, or n/2+1 when full)
    int nb;    // ky/kz extent (2cut+1, or n when full)
    int full;  // 1 when no mode is removed
};

__host__ __device__ __forceinline__ int band_fft_index(const Band& b, int ci) {
    return ci <= b.cut ? ci : b.n - b.nb + ci;
}
__host__ __device__ __forceinline__ int band_compact_index(const Band& b, int fi) {
    // returns -1 when the FFT index is outside the band
    if (b.full) return fi;
    if (fi <= b.cut) return fi;
    if (fi >= b.n - b.cut) return fi - (b.n - b.nb);
    return -1;
}
// signed wavenumber index j of an FFT index
__host__ __device__ __forceinline__ int signed_j(int n, int fi) { return fi <= n / 2 ? fi : fi - n; }

constexpr double MACH_EPSILON = 2.0e-16;  // global_variables.f90:28

struct CudaError : std::runtime_error {
    int status;
    CudaError(const std::string& m, int s) : std::runtime_error(m), status(s) {}
};

#define MLQ_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::mlq::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_),          \
                                   e_ == cudaErrorMemoryAllocation ? MLQ_ERR_OOM : MLQ_ERR_CUDA); \
    } while (0)

}  // namespace mlq
