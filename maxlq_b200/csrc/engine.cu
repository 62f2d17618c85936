// engine.cu -- the precision-independent part of the engine (see engine.cuh):
// bands, twiddles, device memory, reductions, profiling, spectral state ops.
#include "engine_common.cuh"

namespace mlq {

// dealiasing_cutoff_scalar_complex (function_ops.f90:3374, 3391): a mode is
// removed when max_i |K_i| > 2 pi n/(order+1); |K| = 2 pi |j|.  Returns the
// largest |j| kept (n/2 or more means nothing is removed).
int band_cut_for_order(int n, double order) {
    const double kcut = 2.0 * PI_REF * (double)n / (order + 1.0);
    int cut = -1;
    for (int j = 0; j <= n / 2; ++j) {
        const double K = 2.0 * PI_REF * (double)j;
        if (!(std::fabs(K) > kcut)) cut = j;
    }
    return cut;
}

// ----------------------------------------------------------------------------
// EngineBase
// ----------------------------------------------------------------------------
EngineBase::EngineBase(const mlq_params& p) : P(p) {
    n = p.n;
    if (n < 8 || n % 2 != 0) throw CudaError("n must be even and >= 8", MLQ_ERR_BADARG);
    factor_radices(n);
    factor_radices(n / 2);
    if (!p.to_dealias) throw CudaError("toDealias=.false. is not supported", MLQ_ERR_BADARG);
    if (!p.dealias_e_u) throw CudaError("dealiase_if_mult_by_e_u=.false. is not supported", MLQ_ERR_BADARG);
    n3 = (long)n * n * n;
    MLQ_CUDA(cudaSetDevice(p.device));
    MLQ_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    b2 = make_band(band_cut_for_order(n, 2.0));
    bfull = make_band(n / 2);
    if (p.use_e_u_auto)
        use_e_u = p.q < 4.0 - MACH_EPSILON;  // set_e_u_or_just_u (initialize.f90:75-86)
    else
        use_e_u = p.use_e_u != 0;
    // twiddle tables for L = n and n/2 (and every length the plans use)
    std::vector<cpx<double>> pool;
    for (int L : {n, n / 2}) {
        if (tw_off.count(L)) continue;
        tw_off[L] = (int)pool.size();
        for (int k = 0; k < L; ++k) {
            const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)L;
            pool.push_back(mk<double>((double)cosl(a), (double)(-sinl(a))));
        }
    }
    d_tw = (cpx<double>*)dev_alloc(pool.size() * sizeof(cpx<double>));
    // stream-ordered and complete before the first kernel that reads it (a
    // pageable cudaMemcpy may return before its DMA lands, and the engine's
    // stream does not wait for the legacy stream)
    MLQ_CUDA(cudaMemcpyAsync(d_tw, pool.data(), pool.size() * sizeof(cpx<double>), cudaMemcpyHostToDevice, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    d_results = (double*)dev_alloc(NRES * sizeof(double));
    MLQ_CUDA(cudaMemsetAsync(d_results, 0, NRES * sizeof(double), stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    ensure_partials(1 << 20);
    if (const char* e = std::getenv("MLQ_GRAPHS")) graphs_on_ = std::string(e) != "0";
    if (const char* e = std::getenv("MLQ_REUSE")) reuse_on_ = std::string(e) != "0";
    if (const char* e = std::getenv("MLQ_ZMULTI")) multi_zinv_ = std::string(e) != "0";
}

EngineBase::~EngineBase() {
    for (auto& kv : graphs_)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto& a : allocs_) cudaFree(a.first);
    if (stream) cudaStreamDestroy(stream);
}

Band EngineBase::make_band(int cut) const {
    Band b;
    b.n = n;
    if (cut >= n / 2) {
        b.full = 1;
        b.cut = n / 2;
        b.nx = n / 2 + 1;
        b.nb = n;
    } else {
        b.full = 0;
        b.cut = cut;
        b.nx = cut + 1;
        b.nb = 2 * cut + 1;
    }
    return b;
}

FftPlan EngineBase::plan(int L) const {
    FftPlan p;
    std::vector<int> r = factor_radices(L);
    p.L = L;
    p.nst = (int)r.size();
    for (int i = 0; i < p.nst; ++i) p.radix[i] = r[i];
    p.tw_off = tw_off.at(L);
    return p;
}

void* EngineBase::dev_alloc(size_t b) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError("cudaMalloc of " + std::to_string(b) + " bytes failed: " + cudaGetErrorString(e),
                        MLQ_ERR_OOM);
    }
    allocs_.push_back({p, b});
    bytes += (long long)b;
    bytes_peak = std::max(bytes_peak, bytes);
    return p;
}

void EngineBase::free_dev(void* p) {
    auto it = std::find_if(allocs_.begin(), allocs_.end(), [p](const std::pair<void*, size_t>& a) { return a.first == p; });
    if (it != allocs_.end()) {
        ++graph_gen_;  // captured graphs may reference the freed block
        bytes -= (long long)it->second;
        allocs_.erase(it);
        cudaFree(p);
    }
}

SVec* EngineBase::alloc_state() { return dev_alloc(3 * spec_ncomp() * sv_elem()); }


void EngineBase::ensure_partials(long cnt) {
    if (cnt <= partials_cap) return;
    if (d_partials) free_dev(d_partials);
    d_partials = (double*)dev_alloc(cnt * sizeof(double));
    partials_cap = cnt;
}

void EngineBase::finalize(int nblocks, int nr, double scale, int dst, bool accumulate) {
    cudaEvent_t ev = prof_mark();
    finalize_partials_kernel<<<1, RED_THREADS, 0, stream>>>(d_partials, nblocks, nr, scale, d_results, dst,
                                                           accumulate ? 1 : 0);
    launched("finalize", 8.0 * nblocks * nr, ev);
}

void EngineBase::fetch_results() {
    MLQ_CUDA(cudaMemcpyAsync(h_results, d_results, NRES * sizeof(double), cudaMemcpyDeviceToHost, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    if (h_results[NAN_SLOT] != 0.0) {
        // the reference stops the program here (fftwfunction.f90:78-89); the
        // flag is cleared so the context stays usable for a new field
        MLQ_CUDA(cudaMemsetAsync(d_results + NAN_SLOT, 0, sizeof(double), stream));
        MLQ_CUDA(cudaStreamSynchronize(stream));
        h_results[NAN_SLOT] = 0.0;
        throw CudaError("NaN or Inf in a field entering a forward transform", MLQ_ERR_NAN);
    }
}

cudaEvent_t EngineBase::ev_take() {
    if (!evpool_.empty()) {
        cudaEvent_t e = evpool_.back();
        evpool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    MLQ_CUDA(cudaEventCreate(&e));
    return e;
}

cudaEvent_t EngineBase::prof_mark() {
    if (!prof_on) return nullptr;
    cudaEvent_t e = ev_take();
    MLQ_CUDA(cudaEventRecord(e, stream));
    return e;
}

void EngineBase::launched(const char* name, double alg_bytes, cudaEvent_t a) {
    launches += 1;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(e), MLQ_ERR_CUDA);
    if (a) {
        cudaEvent_t b = ev_take();
        MLQ_CUDA(cudaEventRecord(b, stream));
        pend_.push_back(Pend{name ? name : "other", a, b, alg_bytes});
        if (pend_.size() > 4096) prof_flush();
    }
}

void EngineBase::prof_flush() {
    if (pend_.empty()) return;
    MLQ_CUDA(cudaStreamSynchronize(stream));
    for (const Pend& p : pend_) {
        float ms = 0.f;
        MLQ_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
        KStat& k = prof[p.name];
        k.n += 1;
        k.ms += ms;
        k.bytes += p.bytes;
        evpool_.push_back(p.a);
        evpool_.push_back(p.b);
    }
    pend_.clear();
}

std::string EngineBase::prof_report(bool reset) {
    prof_flush();
    std::string s = "{";
    bool first = true;
    for (const auto& kv : prof) {
        char b[256];
        snprintf(b, sizeof(b), "%s\"%s\": [%lld, %.6f, %.1f]", first ? "" : ", ", kv.first.c_str(), kv.second.n,
                 kv.second.ms, kv.second.bytes);
        s += b;
        first = false;
    }
    s += "}";
    if (reset) prof.clear();
    return s;
}

void EngineBase::lincomb(SVec* out, double a, const SVec* x, double b, const SVec* y, double c, const SVec* z) {
    state_written(out);
    SpecGeom g = geom(b2);
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_lincomb_kernel<float2><<<grid_for(3 * g.ncomp, 256), 256, 0, stream>>>(
            g, (float2*)out, a, (const float2*)x, b, (const float2*)y, c, (const float2*)z);
    else
        spec_lincomb_kernel<double2><<<grid_for(3 * g.ncomp, 256), 256, 0, stream>>>(
            g, (double2*)out, a, (const double2*)x, b, (const double2*)y, c, (const double2*)z);
    launched("spec_lincomb", 3.0 * sv_elem() * g.ncomp * (2 + (y ? 1 : 0) + (z ? 1 : 0)), ev);
}

// K = 2 pi j: |K|^2 of a mode with |j|^2 = jsq
static double ksq_of(long jsq) {
    const double twopi = 2.0 * PI_REF;
    return twopi * twopi * (double)jsq;
}

const double* EngineBase::hilbert_table(double order) {
    auto it = htab_.find(order);
    if (it != htab_.end()) return it->second;
    const long m = 3L * b2.cut * b2.cut + 1;
    std::vector<double> h(m);
    for (long j = 0; j < m; ++j) h[j] = 1.0 / (1.0 + std::pow(P.lambda1 * std::sqrt(ksq_of(j)), 2.0 * order));
    double* d = (double*)dev_alloc(m * sizeof(double));
    MLQ_CUDA(cudaMemcpyAsync(d, h.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    htab_[order] = d;
    return d;
}

const double* EngineBase::hweight_table(double order) {
    auto it = hwtab_.find(order);
    if (it != hwtab_.end()) return it->second;
    const long m = 3L * b2.cut * b2.cut + 1;
    std::vector<double> h(m);
    for (long j = 0; j < m; ++j) {
        const double f = 1.0 + std::pow(P.lambda1 * std::sqrt(ksq_of(j)), order);
        h[j] = f * f;
    }
    double* d = (double*)dev_alloc(m * sizeof(double));
    MLQ_CUDA(cudaMemcpyAsync(d, h.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream));
    MLQ_CUDA(cudaStreamSynchronize(stream));
    hwtab_[order] = d;
    return d;
}

static int spec_rows_grid(const SpecGeom& g) { return std::max(1, std::min(g.nb * g.nb, 148 * 16)); }

void EngineBase::retract(SVec* u, double cs, double tau, const SVec* d) {
    const PhysMemo keep = pm_;
    lincomb(u, cs, u, cs * tau, d);
    if (keep.tr && keep.u == (const void*)u && keep.d == (const void*)d && keep.tau == tau) {
        pm_ = keep;
        pm_.u = nullptr;  // the fields describe the old u, no longer stored
        pm_.ls = false;
        pm_.next = u;
        pm_.cs = cs;
    }
}

void EngineBase::transport_retract(SVec* tg, SVec* td, const SVec* g, const SVec* d, SVec* u, double ag,
                                   double bg, double cg, double ad, double bd, double cd, double cs, double tau) {
    const PhysMemo keep = pm_;
    state_written(tg);
    state_written(td);
    state_written(u);
    SpecGeom geo = geom(b2);
    const long nt = 3 * geo.ncomp;
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_transport_kernel<float2><<<grid_for(nt, 256), 256, 0, stream>>>(
            nt, (const float2*)g, (const float2*)d, (float2*)u, (float2*)tg, (float2*)td, ag, bg, cg, ad, bd, cd, cs,
            cs * tau);
    else
        spec_transport_kernel<double2><<<grid_for(nt, 256), 256, 0, stream>>>(
            nt, (const double2*)g, (const double2*)d, (double2*)u, (double2*)tg, (double2*)td, ag, bg, cg, ad, bd, cd,
            cs, cs * tau);
    launched("spec_lincomb", (double)sv_elem() * nt * 6, ev);
    if (keep.tr && keep.u == (const void*)u && keep.d == (const void*)d && keep.tau == tau) {
        pm_ = keep;
        pm_.u = nullptr;  // the fields describe the old u, no longer stored
        pm_.ls = false;
        pm_.next = u;
        pm_.cs = cs;
    }
}

void EngineBase::hilbert(SVec* f, double order) {
    state_written(f);
    SpecGeom g = geom(b2);
    const double* t = hilbert_table(order);
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_hilbert_leray_kernel<float2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (float2*)f, t, 1.0, 0);
    else
        spec_hilbert_leray_kernel<double2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (double2*)f, t, 1.0, 0);
    launched("spec_hilbert", 6.0 * sv_elem() * g.ncomp, ev);
}

void EngineBase::leray(SVec* f) {
    state_written(f);
    SpecGeom g = geom(b2);
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_hilbert_leray_kernel<float2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (float2*)f, nullptr, 1.0, 1);
    else
        spec_hilbert_leray_kernel<double2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (double2*)f, nullptr, 1.0, 1);
    launched("spec_leray", 6.0 * sv_elem() * g.ncomp, ev);
}

void EngineBase::hilbert_leray(SVec* f, double order, double scale) {
    state_written(f);
    SpecGeom g = geom(b2);
    const double* t = hilbert_table(order);
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_hilbert_leray_kernel<float2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (float2*)f, t, scale, 1);
    else
        spec_hilbert_leray_kernel<double2><<<spec_rows_grid(g), 128, 0, stream>>>(g, (double2*)f, t, scale, 1);
    launched("spec_hilbert_leray", 6.0 * sv_elem() * g.ncomp, ev);
}

void EngineBase::hilbert_leray_pair_dots(SVec* f1, SVec* f2, double order, double s2, double out[2]) {
    state_written(f1);
    state_written(f2);
    SpecGeom g = geom(b2);
    const double* t = hilbert_table(order);
    const double* hw = hweight_table(1.5 - 1.0 / P.q);  // (3/2)-(1/q), function_ops.f90:3467
    const int grid = spec_rows_grid(g);
    ensure_partials((long)grid * 2);
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_hilbert_leray_pair_dot_kernel<float2><<<grid, 128, 0, stream>>>(g, (float2*)f1, 1.0, (float2*)f2, s2, t,
                                                                              hw, d_partials);
    else
        spec_hilbert_leray_pair_dot_kernel<double2><<<grid, 128, 0, stream>>>(g, (double2*)f1, 1.0, (double2*)f2,
                                                                               s2, t, hw, d_partials);
    launched("spec_hilbert_leray", 2 * 6.0 * sv_elem() * g.ncomp, ev);
    finalize(grid, 2, 1.0, 200);
    fetch_results();
    out[0] = h_results[200];
    out[1] = h_results[201];
}

void EngineBase::direction(SVec* gv, double sg, SVec* d, double beta, const SVec* td) {
    state_written(gv);
    state_written(d);
    SpecGeom g = geom(b2);
    const long nt = 3 * g.ncomp;
    cudaEvent_t ev = prof_mark();
    if (state32_)
        spec_direction_kernel<float2><<<grid_for(nt, 256), 256, 0, stream>>>(nt, (float2*)gv, sg, (float2*)d,
                                                                            td ? beta : 0.0, (const float2*)td);
    else
        spec_direction_kernel<double2><<<grid_for(nt, 256), 256, 0, stream>>>(nt, (double2*)gv, sg, (double2*)d,
                                                                             td ? beta : 0.0, (const double2*)td);
    launched("spec_lincomb", (double)sv_elem() * nt * (3 + (td ? 1 : 0)), ev);
}

// ---- spectral inner products ----
using DotLaunch = void (*)(int, cudaStream_t, const SpecDotArgs&);
template <class K>
static int dot_resident(K kernel) {
    int per_sm = 0, dev = 0, sms = 0;
    MLQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, RED_THREADS, 0));
    MLQ_CUDA(cudaGetDevice(&dev));
    MLQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return std::max(1, per_sm) * sms;
}
template <typename V>
static void launch_dot_generic(int grid, cudaStream_t s, const SpecDotArgs& a) {
    spec_dot_kernel<V><<<grid, RED_THREADS, 0, s>>>(a);
}
template <typename V, int NV, int NP, unsigned long long PAT>
static void launch_dot_fixed(int grid, cudaStream_t s, const SpecDotArgs& a) {
    spec_dot_fixed_kernel<V, NV, NP, PAT><<<grid, RED_THREADS, 0, s>>>(a);
}
// operand pattern of pair p: vector indices ia, ib
constexpr unsigned long long dot_pp(int p, int ia, int ib) {
    return (unsigned long long)(ia | (ib << 3)) << (6 * p);
}
constexpr unsigned long long dot_ax(int xi, int yi) {
    return ((unsigned long long)xi << 48) | ((unsigned long long)yi << 51);
}
struct DotVariant {
    int nv, np;
    unsigned long long pat;
    DotLaunch fn[2];  // FP32, FP64 state
    int resident[2];
};
template <int NV, int NP, unsigned long long PAT>
static DotVariant dot_variant() {
    return {NV,
            NP,
            PAT,
            {launch_dot_fixed<float2, NV, NP, PAT>, launch_dot_fixed<double2, NV, NP, PAT>},
            {dot_resident(spec_dot_fixed_kernel<float2, NV, NP, PAT>),
             dot_resident(spec_dot_fixed_kernel<double2, NV, NP, PAT>)}};
}
// The operand patterns the programs use, each with its own kernel:
//   the CG update (g <- g - alpha c, then <g,c>_H, |div g|^2, <g,g>_H, <u,u>_H,
//     <g,Tg0>_H, <g0,g0>_H, <g,Td0>_H, <Td0,Td0>_H over c, u, Tg0, g0, Td0, g);
//   the transport's two products <c, g>, <c, d>; one pair of a vector with
//   itself or with another.
constexpr unsigned long long DOT_CG = dot_pp(0, 5, 0) | dot_pp(1, 5, 5) | dot_pp(2, 5, 5) | dot_pp(3, 1, 1) |
                                      dot_pp(4, 5, 2) | dot_pp(5, 3, 3) | dot_pp(6, 5, 4) | dot_pp(7, 4, 4) |
                                      dot_ax(5, 0);
constexpr unsigned long long DOT_TRANSPORT = dot_pp(0, 0, 1) | dot_pp(1, 0, 2);

void EngineBase::dots(const SpecDotPair* pairs, int np, double* out, SVec* ax_out, const SVec* ax_x, double ax_a,
                      const SVec* ax_y) {
    if (np < 1 || np > 8) throw CudaError("dots: 1 to 8 pairs per call", MLQ_ERR_BADARG);
    SpecDotArgs a;
    a.g = geom(b2);
    for (int i = 0; i < np; ++i) a.pr[i] = pairs[i];
    a.npairs = np;
    if (ax_out) {
        state_written(ax_out);
        a.ax_out = ax_out;
        a.ax_x = ax_x;
        a.ax_y = ax_y;
        a.ax_a = ax_a;
    }
    bool need_h = false;
    for (int i = 0; i < np; ++i) need_h |= pairs[i].kind == 1;
    a.hwtab = need_h ? hweight_table(1.5 - 1.0 / P.q) : nullptr;  // (3/2)-(1/q), function_ops.f90:3467
    // the distinct vectors (update operands first, ax_out moved last) and
    // the operand pattern over them
    std::vector<const void*> order;
    auto add = [&](const void* p) {
        if (std::find(order.begin(), order.end(), p) == order.end()) order.push_back(p);
    };
    if (ax_out) {
        add(ax_x);
        add(ax_y);
    }
    for (int i = 0; i < np; ++i) {
        add(pairs[i].a);
        if (pairs[i].kind < 2) add(pairs[i].b);
    }
    if (ax_out) {
        const auto it = std::find(order.begin(), order.end(), (const void*)ax_out);
        if (it != order.end()) {
            order.erase(it);
            order.push_back(ax_out);
            a.ax_last = 1;
        }
    }
    auto slot = [&](const void* p) { return (int)(std::find(order.begin(), order.end(), p) - order.begin()); };
    const int nv = (int)order.size();
    unsigned long long pat = 0;
    for (int i = 0; i < np; ++i) {
        const int ia = slot(pairs[i].a);
        pat |= dot_pp(i, ia, pairs[i].kind < 2 ? slot(pairs[i].b) : ia);
    }
    if (ax_out) pat |= dot_ax(slot(ax_x), slot(ax_y));
    for (int v = 0; v < nv && v < 8; ++v) a.vec[v] = order[v];
    // as many blocks as are resident at once: the reduction is latency-bound
    // (thread-safe one-time initialisation; every device here is a B200)
    struct Table {
        std::vector<DotVariant> fixed;
        DotLaunch generic[2];
        int generic_resident[2];
    };
    static const Table tab = [] {
        Table t;
        t.fixed = {dot_variant<6, 8, DOT_CG>(), dot_variant<3, 2, DOT_TRANSPORT>(), dot_variant<1, 1, 0>(),
                   dot_variant<2, 1, dot_pp(0, 0, 1)>()};
        t.generic[0] = launch_dot_generic<float2>;
        t.generic[1] = launch_dot_generic<double2>;
        t.generic_resident[0] = dot_resident(spec_dot_kernel<float2>);
        t.generic_resident[1] = dot_resident(spec_dot_kernel<double2>);
        return t;
    }();
    const int w = state32_ ? 0 : 1;
    const DotVariant* fv = nullptr;
    for (const DotVariant& d : tab.fixed)
        if (d.nv == nv && d.np == np && d.pat == pat) fv = &d;
    const int grid = grid_for(a.g.ncomp, RED_THREADS, fv ? fv->resident[w] : tab.generic_resident[w]);
    ensure_partials((long)grid * 8);
    a.partials = d_partials;
    cudaEvent_t ev = prof_mark();
    (fv ? fv->fn[w] : tab.generic[w])(grid, stream, a);
    // vectors read (ax_out only when it is an update operand) and written
    const bool out_read = ax_out && (ax_out == ax_x || ax_out == ax_y);
    const int nread = nv - ((a.ax_last && !out_read) ? 1 : 0);
    launched("spec_dot", 3.0 * sv_elem() * a.g.ncomp * (nread + (ax_out ? 1 : 0)), ev);
    finalize(grid, 8, 1.0, 200);
    fetch_results();
    for (int i = 0; i < np; ++i) out[i] = h_results[200 + i];
}

void EngineBase::zeroth(const SVec* f, double out[3]) {
    double2 h[3];
    float2 hf[3];
    for (int c = 0; c < 3; ++c) {
        if (state32_)
            MLQ_CUDA(cudaMemcpyAsync(&hf[c], scomp(f, c), sizeof(float2), cudaMemcpyDeviceToHost, stream));
        else
            MLQ_CUDA(cudaMemcpyAsync(&h[c], scomp(f, c), sizeof(double2), cudaMemcpyDeviceToHost, stream));
    }
    MLQ_CUDA(cudaStreamSynchronize(stream));
    const double s = (double)n3;  // unnormalised k=0 coefficient (function_ops.f90:3084-3086)
    for (int c = 0; c < 3; ++c) out[c] = (state32_ ? (double)hf[c].x : h[c].x) * s;
}

}  // namespace mlq
