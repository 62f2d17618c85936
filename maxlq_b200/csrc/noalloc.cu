// noalloc.cu -- dealias_scalar without any device allocation.
//
// mlq_dealias_scalar_noalloc runs the same pass kernels as mlq_dealias_scalar
// (x stage r2c, y FFT, z round trip with the cube mask, inverse y, inverse x)
// but takes every byte of device memory it needs -- the field, the two
// pipeline intermediates, the reduction partials and the twiddle tables --
// from one file-scope static __device__ array sized for N <= MLQ_NOALLOC_MAX_N.
// It is for callers that cannot allocate device memory: it needs no context
// (mlq_init allocates), and calls neither cudaMalloc nor cudaFree nor any
// library routine that allocates.
#include <cmath>
#include <cstdio>

#include "functors.cuh"
#include "kernels.cuh"

namespace mlq {
int band_cut_for_order(int n, double order);
}

using namespace mlq;

namespace {

constexpr int NMAX = MLQ_NOALLOC_MAX_N;
constexpr size_t PHYS_BYTES = (size_t)NMAX * NMAX * NMAX * sizeof(double);
constexpr size_t LINE_CPX = (size_t)NMAX * NMAX * (NMAX / 2 + 1);  // n * n * (n/2+1) complex
constexpr size_t XS_BYTES = LINE_CPX * sizeof(cpx<double>);
constexpr size_t YS_BYTES = LINE_CPX * sizeof(cpx<double>);
constexpr size_t PART_DOUBLES = 4096 * MAX_RED;
constexpr size_t TW_CPX = NMAX + NMAX / 2;
constexpr size_t OFF_PHYS = 0;
constexpr size_t OFF_XS = OFF_PHYS + PHYS_BYTES;
constexpr size_t OFF_YS = OFF_XS + XS_BYTES;
constexpr size_t OFF_PART = OFF_YS + YS_BYTES;
constexpr size_t OFF_TW = OFF_PART + PART_DOUBLES * sizeof(double);
constexpr size_t SCRATCH_BYTES = OFF_TW + TW_CPX * sizeof(cpx<double>);
static_assert(OFF_XS % 256 == 0 && OFF_YS % 256 == 0 && OFF_PART % 256 == 0 && OFF_TW % 256 == 0,
              "scratch regions stay 256-byte aligned");

// The scratch.  Its name in host code is only a handle for
// cudaGetSymbolAddress; kernels receive the device address obtained that way.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

// The device address of the scratch in the calling thread's current context.
// It is looked up on every call (a cheap runtime query): a symbol's address
// belongs to a CUDA context, and a caller may switch contexts on a device
// (another runtime's driver-API context, or a cudaDeviceReset) between calls.
cudaError_t scratch_address(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

bool radix_ok(int L) {
    int m = L;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    return m == 1;
}

FftPlan make_plan(int L, int tw_off) {
    FftPlan p;
    p.L = L;
    p.nst = 0;
    p.tw_off = tw_off;
    int m = L;
    const int order[4] = {16, 8, 4, 2};
    for (int r : order)
        while (m % r == 0 && m > 1) {
            p.radix[p.nst++] = r;
            m /= r;
        }
    while (m % 3 == 0) {
        p.radix[p.nst++] = 3;
        m /= 3;
    }
    return p;
}

int fail(int status, const char* msg) {
    fprintf(stderr, "mlq_dealias_scalar_noalloc: %s\n", msg);
    return status;
}

int launch_failed(const char* kernel, cudaError_t e) {
    char m[200];
    snprintf(m, sizeof(m), "launch of the %s kernel failed: %s", kernel, cudaGetErrorString(e));
    return fail(MLQ_ERR_CUDA, m);
}

}  // namespace

extern "C" int mlq_dealias_scalar_noalloc(double* g, int n, double order) {
    if (!g) return fail(MLQ_ERR_BADARG, "null field");
    if (n < 8 || n % 2 != 0 || !radix_ok(n))
        return fail(MLQ_ERR_BADARG, "n must be even, >= 8 and of the form 2^a 3^b");
    if (n > NMAX) {
        char m[160];
        snprintf(m, sizeof(m), "n=%d exceeds the static scratch of this entry point (n <= %d); use mlq_dealias_scalar",
                 n, NMAX);
        return fail(MLQ_ERR_BADARG, m);
    }
    if (!std::isfinite(order)) return fail(MLQ_ERR_BADARG, "order must be finite");
    const int cut = band_cut_for_order(n, order);
    if (cut < 0) return fail(MLQ_ERR_BADARG, "order < -1 keeps no mode; dealias orders are >= 0");
    if (cut >= n / 2) return MLQ_OK;  // the mask removes nothing (order <= 1), as mlq_dealias_scalar
    // an error left pending by earlier work of the caller is reported as such,
    // not blamed on a launch below
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char m[200];
        snprintf(m, sizeof(m), "a CUDA error was pending before this call: %s", cudaGetErrorString(e));
        return fail(MLQ_ERR_CUDA, m);
    }
    unsigned char* base = nullptr;
    e = scratch_address(&base);
    if (e != cudaSuccess) return fail(MLQ_ERR_CUDA, cudaGetErrorString(e));

    double* phys = reinterpret_cast<double*>(base + OFF_PHYS);
    cpx<double>* xs = reinterpret_cast<cpx<double>*>(base + OFF_XS);
    cpx<double>* ys = reinterpret_cast<cpx<double>*>(base + OFF_YS);
    double* partials = reinterpret_cast<double*>(base + OFF_PART);
    cpx<double>* tw = reinterpret_cast<cpx<double>*>(base + OFF_TW);

    // band of the cube cut (function_ops.f90:3374-3391)
    Band b;
    b.n = n;
    b.full = 0;
    b.cut = cut;
    b.nx = cut + 1;
    b.nb = 2 * cut + 1;
    const int h = n / 2;
    const long n3 = (long)n * n * n;

    // twiddles W_n then W_{n/2}; rewritten by every call since n may change
    cpx<double> htw[TW_CPX];
    for (int k = 0; k < n; ++k) {
        const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
        htw[k] = mk<double>((double)cosl(a), (double)(-sinl(a)));
    }
    for (int k = 0; k < h; ++k) {
        const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)h;
        htw[n + k] = mk<double>((double)cosl(a), (double)(-sinl(a)));
    }
    if ((e = cudaMemcpy(tw, htw, (size_t)(n + h) * sizeof(cpx<double>), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(phys, g, n3 * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(MLQ_ERR_CUDA, cudaGetErrorString(e));

    const FftPlan plan_n = make_plan(n, 0), plan_h = make_plan(h, n);
    int lx = 8;
    while (lx > 1 && ((long)n * n) % lx != 0) lx /= 2;
    const int tx = 16;

    // x stage (r2c, keep kx <= cut)
    XFwdArgs<double> xa;
    xa.n = n;
    xa.nx = b.nx;
    xa.lx = lx;
    xa.in[0] = phys;
    xa.out[0] = xs;
    xa.plan_half = plan_h;
    xa.tw_n_off = 0;
    xa.tw = tw;
    xa.partials = partials;
    xfwd_kernel<double, FCopy><<<(unsigned)((long)n * n / lx), 256, 2 * lx * h * sizeof(cpx<double>)>>>(xa, FCopy{});
    if ((e = cudaGetLastError()) != cudaSuccess) return launch_failed("x stage (r2c)", e);
    // y forward (keep |ky| <= cut)
    YArgs<double> ya;
    ya.n = n;
    ya.nx = b.nx;
    ya.tx = tx;
    ya.band = b;
    ya.in[0] = xs;
    ya.out[0] = ys;
    ya.plan = plan_n;
    ya.tw = tw;
    const size_t ysm = 2 * (size_t)n * tx * sizeof(cpx<double>);
    dim3 yg((b.nx + tx - 1) / tx, n, 1);
    ypass_kernel<-1, double><<<yg, 256, ysm>>>(ya);
    if ((e = cudaGetLastError()) != cudaSuccess) return launch_failed("y forward", e);
    // z round trip with the mask and the 1/N^3 of the forward transform
    ZFwdArgs<double> za;
    za.n = n;
    za.nx = b.nx;
    za.tx = tx;
    za.band = b;
    ZFwdOp op = {};
    op.in = ys;
    op.ys_out = ys;
    op.sym = SYM_ONE;
    op.red_self = -1;
    for (int r = 0; r < 3; ++r) op.red_with_slot[r] = -1;
    za.op[0] = op;
    za.plan = plan_n;
    za.tw = tw;
    za.partials = partials;
    za.norm = 1.0 / (double)n3;
    dim3 zg((b.nx + tx - 1) / tx, b.nb, 1);
    if ((size_t)zg.x * zg.y * MAX_RED > PART_DOUBLES) return fail(MLQ_ERR_BADARG, "partials scratch too small");
    zfwd_kernel<double><<<zg, 256, ysm>>>(za);
    if ((e = cudaGetLastError()) != cudaSuccess) return launch_failed("z round trip", e);
    // y inverse, x inverse (c2r) back into the field
    YArgs<double> yb = ya;
    yb.in[0] = ys;
    yb.out[0] = xs;
    ypass_kernel<+1, double><<<yg, 256, ysm>>>(yb);
    if ((e = cudaGetLastError()) != cudaSuccess) return launch_failed("y inverse", e);
    XInvArgs<double> xb;
    xb.n = n;
    xb.nx_in = b.nx;
    xb.lx = lx;
    xb.in[0] = xs;
    xb.out[0] = phys;
    xb.plan_half = plan_h;
    xb.tw_n_off = 0;
    xb.tw = tw;
    dim3 xg((unsigned)((long)n * n / lx), 1);
    xinv_kernel<double><<<xg, 256, (size_t)(3 * h + 1) * lx * sizeof(cpx<double>)>>>(xb);
    if ((e = cudaGetLastError()) != cudaSuccess) return launch_failed("x inverse (c2r)", e);
    if ((e = cudaMemcpy(g, phys, n3 * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return fail(MLQ_ERR_CUDA, cudaGetErrorString(e));
    return MLQ_OK;
}
