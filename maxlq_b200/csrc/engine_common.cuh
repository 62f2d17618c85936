// engine_common.cuh -- host helpers shared by the engine's translation units.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <typeinfo>

#include <cxxabi.h>

#include "engine.cuh"

namespace mlq {

static const double PI_REF = 4.0 * std::atan2(1.0, 1.0);  // initialize.f90:164


static std::vector<int> factor_radices(int L) {
    std::vector<int> r;
    int m = L;
    while (m % 16 == 0 && m > 1) { r.push_back(16); m /= 16; }
    while (m % 8 == 0) { r.push_back(8); m /= 8; }
    while (m % 4 == 0) { r.push_back(4); m /= 4; }
    while (m % 2 == 0) { r.push_back(2); m /= 2; }
    while (m % 3 == 0) { r.push_back(3); m /= 3; }
    if (m != 1) throw CudaError("FFT length must be 2^a 3^b", MLQ_ERR_BADARG);
    return r;
}

// raise the dynamic shared memory limit of each kernel once (per device
// function address: kernels of equal type are distinct entries)
// (contexts may be driven from several host threads at once)
inline std::mutex& smem_attr_mutex() {
    static std::mutex m;
    return m;
}
template <typename K>
static void allow_smem(K kernel) {
    static std::set<const void*> done;
    const void* key = reinterpret_cast<const void*>(kernel);
    std::lock_guard<std::mutex> lock(smem_attr_mutex());
    if (done.insert(key).second) {
        // the opt-in per-block limit less the kernel's static shared memory
        int dev = 0, optin = 0;
        cudaFuncAttributes fa{};
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     optin - (int)fa.sharedSizeBytes);
        if (e != cudaSuccess) throw CudaError(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e), MLQ_ERR_CUDA);
    }
}

// f(std::integral_constant<int, n>) for the sizes with compile-time kernels
template <class Fn>
static bool dispatch_n(int n, Fn&& f) {
    switch (n) {
        case 64: f(std::integral_constant<int, 64>{}); return true;
        case 128: f(std::integral_constant<int, 128>{}); return true;
        case 256: f(std::integral_constant<int, 256>{}); return true;
        case 512: f(std::integral_constant<int, 512>{}); return true;
        case 1024: f(std::integral_constant<int, 1024>{}); return true;
        default: return false;
    }
}

// profile key of an x-stage launch: "x_fwd", or "x_fwd:<functor>" in detail mode
template <class F>
static const char* xfwd_name(bool detail) {
    static const std::string name = [] {
        int st = 0;
        char* d = abi::__cxa_demangle(typeid(F).name(), nullptr, nullptr, &st);
        std::string s = std::string("x_fwd:") + (st == 0 && d ? d : typeid(F).name());
        std::free(d);
        const std::string ns = "mlq::";
        for (size_t p; (p = s.find(ns)) != std::string::npos;) s.erase(p, ns.size());
        return s;
    }();
    return detail ? name.c_str() : "x_fwd";
}

static int grid_for(long work, int threads, int cap = 148 * 8) {
    long g = (work + threads - 1) / threads;
    return (int)std::max(1L, std::min<long>(g, cap));
}

}  // namespace mlq
