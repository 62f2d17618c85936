// engine.cuh -- the B200 engine behind the C ABI.
//
// State: every CG vector (u, d, gradients, transported vectors) lives on the
// device as pruned FP64 Fourier coefficients of the 2/3-dealiased band
// (the only modes a band-limited field has).  Work: each operator of the
// reference is a pipeline of pass kernels (kernels.cuh) in precision T with
// the pointwise products fused into the x stage (functors.cuh) and the
// spectral multiplies, masks and Parseval reductions in the z stage.
#pragma once

#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "functors.cuh"
#include "kernels.cuh"
#include "regfft.cuh"
#include "cfft.cuh"
#include "linesearch.cuh"

namespace mlq {

// launchers of the device line search's kernels (lsdev.cu)
void ls_launch_coef(LsDevState* s, const double* results, const double* partials, int nblocks, const LsAnchorSet& an,
                    cudaStream_t st);
void ls_launch_ctrl(LsDevState* s, cudaGraphConditionalHandle h_loop, cudaGraphConditionalHandle h_chk,
                    cudaStream_t st);
void ls_launch_check(LsDevState* s, const double* partials, int nblocks, cudaGraphConditionalHandle h_fft,
                     cudaStream_t st);
void ls_launch_fft(LsDevState* s, const double* r, cudaStream_t st);

// A state vector: three components of nb*nb*nx Fourier coefficients of band
// b2, stored as double2 (FP64 path) or float2 (the mixed path's FP32 state);
// every operation on it computes in FP64.  Components are addressed with
// EngineBase::scomp, never by pointer arithmetic.
using SVec = void;

int band_cut_for_order(int n, double order);

struct PhysField;  // fwd

// Engine-independent part (device, stream, params, bands, twiddles).
class EngineBase {
   public:
    explicit EngineBase(const mlq_params& p);
    virtual ~EngineBase();

    mlq_params P;
    int n;
    long n3;
    Band b2;            // P2 band: the state band
    Band bfull;         // no cut
    cudaStream_t stream = nullptr;
    long long launches = 0;
    long long bytes = 0;
    bool use_e_u = false;

    // twiddles: pool of W_L tables
    cpx<double>* d_tw = nullptr;
    std::map<int, int> tw_off;  // L -> offset
    FftPlan plan(int L) const;

    // device reductions
    double* d_partials = nullptr;
    long partials_cap = 0;
    double* d_results = nullptr;  // 256 slots
    static constexpr int NRES = 256;
    // result slot the forward transforms set when they meet a non-finite
    // value; fetch_results() turns it into MLQ_ERR_NAN
    static constexpr int NAN_SLOT = NRES - 1;
    double h_results[NRES];
    void fetch_results();  // sync + copy all slots; throws MLQ_ERR_NAN if a NaN was seen

    // FP64 state spectra (3 components each) of band b2
    long spec_ncomp() const { return (long)b2.nb * b2.nb * b2.nx; }
    // state storage: FP32 in the mixed path (MLQ_STATE_F64=1 keeps FP64)
    bool state32_ = false;
    size_t sv_elem() const { return state32_ ? sizeof(float2) : sizeof(double2); }
    int sf64() const { return state32_ ? 0 : 1; }  // the f64 flag of z-stage sources/outputs
    SVec* scomp(SVec* v, int c) const { return (char*)v + (size_t)c * spec_ncomp() * sv_elem(); }
    const SVec* scomp(const SVec* v, int c) const { return (const char*)v + (size_t)c * spec_ncomp() * sv_elem(); }
    SVec* alloc_state();
    void free_dev(void* p);
    void* dev_alloc(size_t bytes);
    SpecGeom geom(const Band& b) const {
        SpecGeom g;
        g.n = n;
        g.nx = b.nx;
        g.nb = b.nb;
        g.band = b;
        g.ncomp = (long)b.nb * b.nb * b.nx;
        return g;
    }
    Band make_band(int cut) const;

    // spectral state ops (FP64)
    void lincomb(SVec* out, double a, const SVec* x, double b = 0, const SVec* y = nullptr, double c = 0,
                 const SVec* z = nullptr);
    void hilbert(SVec* f, double order);
    void leray(SVec* f);
    // f <- leray(hilbert(scale * f, order)) in one pass
    void hilbert_leray(SVec* f, double order, double scale = 1.0);
    // tables over |j|^2 of the band b2: Hilbert symbol and H_l inner-product weight
    std::map<double, double*> htab_, hwtab_;
    const double* hilbert_table(double order);
    const double* hweight_table(double order);
    // up to 8 vector inner products; kinds 0 L2, 1 H_l, 2 div energy,
    // 3 curl energy sum |K x a|^2, 4 Laplacian energy sum |K|^4 |a|^2
    // (kinds 2-4 read only a)
    // pairs' inner products; optionally ax_out <- ax_x + ax_a ax_y first, in
    // the same pass (the pairs may name ax_out)
    void dots(const SpecDotPair* pairs, int np, double* out, SVec* ax_out = nullptr,
              const SVec* ax_x = nullptr, double ax_a = 0.0, const SVec* ax_y = nullptr);
    // hilbert_leray of f1 (scale 1) and f2 (scale s2), then out = {<f2, f1>_H, <f2, f2>_H}
    void hilbert_leray_pair_dots(SVec* f1, SVec* f2, double order, double s2, double out[2]);
    // g <- sg g, d <- g + beta td (td null: d <- g)
    void direction(SVec* g, double sg, SVec* d, double beta, const SVec* td);
    void zeroth(const SVec* f, double out[3]);

    // ---- diagnostics (maxdLpdt.f90:263-299, optimization.f90:119-123, 377-384) ----
    // calculate_spectral_data (function_ops.f90:2614-2677) of the state
    // spectra u: out[0..n) = kk_max = 2 pi (i+1), out[n..2n) = the shell
    // energies of fftfwd(u), scaled by <u,u>/(2 pi sum) when normalize
    void spectrum(const SVec* u, bool normalize, double* out);
    // calc_global_summed_enstrophy (2449-2467): 1/2 ||curl u||^2
    double enstrophy(const SVec* u);
    // per-shell lists of the band's modes (|K| in (2 pi i, 2 pi (i+1)]),
    // built once; the shell sums then run in a fixed order
    int* d_shell_modes_ = nullptr;
    int* d_shell_off_ = nullptr;

    void finalize(int nblocks, int nr, double scale, int dst, bool accumulate = false);
    // The state spectrum whose u and grad u the physical fields 0..11 hold
    // (set by the gradient program; cleared by any write to that spectrum or
    // to those fields), so the line-search setup of the same iteration can
    // reuse them instead of transforming again.
    const void* pu_of_ = nullptr;
    // Physical fields the line search leaves for the transport and the next
    // gradient program (resident mode).  ls: after the line-search setup,
    // phys(iu..iu+2) = u, phys(idu..idu+8) = grad u, and the fields 63..65,
    // 75..83 hold d and grad d, for the spectra u, d.  tr: after a transport
    // (or Lq norm) at w = u + tau d formed from them, phys 0..2 = w while
    // idu and 75..83 still hold grad u and grad d.  retract() then records
    // that the state spectrum `next` holds cs * w, and the next gradient
    // program forms u and grad u pointwise instead of transforming them.
    // sac: the transport also left P2(|w|^2), P2(g^2) (physical 18, 19 and
    // work spectrum 1) and P2(|w|^2 w) (c_tmp_) at q = 4, which the gradient
    // program at cs w scales by cs^2 and cs^3.  Cleared by a write to
    // physical fields 0..11, 18, 19 or 60..83 and by a write to any of the
    // spectra.
    struct PhysMemo {
        const void* u = nullptr;
        const void* d = nullptr;
        const void* next = nullptr;
        int iu = -1, idu = -1;
        bool ls = false, tr = false, sac = false;
        double tau = 0.0, cs = 0.0;
    } pm_;
    // the state spectrum whose S = P2(|u|^2) the physical field 18 and a work
    // spectrum hold (set by the gradient program), for the line-search setup
    const void* ws_of_ = nullptr;
    void state_written(const void* p) {
        if (p == pu_of_) pu_of_ = nullptr;
        if (p == ws_of_) ws_of_ = nullptr;
        if (p && (p == pm_.u || p == pm_.d || p == pm_.next)) pm_ = PhysMemo{};
    }
    // u <- cs (u + tau d), keeping the transport's physical fields of
    // u + tau d for the next gradient program
    void retract(SVec* u, double cs, double tau, const SVec* d);
    // the vector transport's outputs tg = ag g + bg u + cg d, td = ad d + bd u
    // + cd d and then the retraction u <- cs (u + tau d), in one pass
    void transport_retract(SVec* tg, SVec* td, const SVec* g, const SVec* d, SVec* u, double ag,
                           double bg, double cg, double ad, double bd, double cd, double cs, double tau);
    void ensure_partials(long n);
    // Count a launch and surface launch-configuration errors immediately.
    // With profiling on, `a` is the event recorded before the launch; the
    // launch's device time and its algorithmic bytes (compulsory reads +
    // writes) are accumulated per kernel name.
    void launched(const char* name = nullptr, double alg_bytes = 0.0, cudaEvent_t a = nullptr);
    cudaEvent_t prof_mark();
    bool prof_on = false;

    // ---- CUDA graphs of fixed launch sequences ----
    // as_graph(name, key, body): the first call with a key runs body() as is
    // (lazy allocations, attributes), the second captures it into a graph,
    // later calls with the same key launch the graph.  body() may issue only
    // stream-ordered work.  Freeing device memory drops every graph (they may
    // hold the pointers); profiling runs bodies directly.  MLQ_GRAPHS=0 turns
    // graphs off.
    struct ProgGraph {
        std::vector<const void*> key;
        long gen = -1;
        int seen = 0;
        bool disabled = false;
        long long nlaunch = 0;
        cudaGraphExec_t exec = nullptr;
    };
    std::map<std::string, ProgGraph> graphs_;
    long graph_gen_ = 0;
    bool graphs_on_ = true;
    // the exact-arithmetic reuse paths (fields formed pointwise or from the
    // line search's coefficients, W as half-gradients of |phi|^2); MLQ_REUSE=0
    // runs every program in its plain transform sequence instead
    bool reuse_on_ = true;
    // single-source z inverse launches grouped by source (one load per
    // column for a field and its derivatives); MLQ_ZMULTI=0 turns it off
    bool multi_zinv_ = true;
    long long graph_launches_ = 0;  // graphs launched (replays)
    template <class Fn>
    void as_graph(const std::string& name, const std::vector<const void*>& key, Fn&& body);
    bool prof_detail = false;  // x-stage launches keyed by functor as well
    struct KStat {
        long long n = 0;
        double ms = 0.0, bytes = 0.0;
    };
    std::map<std::string, KStat> prof;
    void prof_flush();
    std::string prof_report(bool reset);
    virtual std::string kernel_config() const { return "{}"; }

   private:
    struct Pend {
        const char* name;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pend> pend_;
    std::vector<cudaEvent_t> evpool_;

   public:
    cudaEvent_t ev_take();  // from the engine's pool of events
    void ev_give(cudaEvent_t e) { evpool_.push_back(e); }

    std::vector<std::pair<void*, size_t>> allocs_;
    long long bytes_peak = 0;  // most device bytes held at once
};

template <class Fn>
void EngineBase::as_graph(const std::string& name, const std::vector<const void*>& key, Fn&& body) {
    if (!graphs_on_ || prof_on) {
        body();
        return;
    }
    // one cached graph per (name, key): callers alternate between buffers
    std::string id = name;
    for (const void* k : key) id += ":" + std::to_string(reinterpret_cast<uintptr_t>(k));
    if (graphs_.size() > 32 && !graphs_.count(id)) {
        for (auto& kv : graphs_)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        graphs_.clear();
    }
    ProgGraph& g = graphs_[id];
    if (g.key != key || g.gen != graph_gen_) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.key = key;
        g.gen = graph_gen_;
        g.seen = 0;
    }
    if (g.exec) {
        MLQ_CUDA(cudaGraphLaunch(g.exec, stream));
        launches += g.nlaunch;
        ++graph_launches_;
        return;
    }
    if (g.disabled || g.seen++ == 0) {
        body();
        return;
    }
    const long long l0 = launches;
    MLQ_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    bool ok = true;
    try {
        body();
    } catch (...) {
        ok = false;
    }
    cudaGraph_t gr = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(stream, &gr);
    if (ok && ec == cudaSuccess && gr) {
        const cudaError_t ei = cudaGraphInstantiate(&g.exec, gr, 0);
        cudaGraphDestroy(gr);
        if (ei == cudaSuccess && g.gen == graph_gen_) {
            g.nlaunch = launches - l0;
            launches = l0;
            MLQ_CUDA(cudaGraphLaunch(g.exec, stream));
            launches += g.nlaunch;
            ++graph_launches_;
            return;
        }
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    } else if (gr) {
        cudaGraphDestroy(gr);
    }
    // capture failed (for instance an allocation inside body): run directly
    cudaGetLastError();
    g.disabled = true;
    launches = l0;
    body();
}

// A physical-space power field |u|^k as computed by calc_uk.
struct PowField {
    enum Kind { ONE, RAW, BAND } kind = ONE;
    double k = 0;
    int phys = -1;       // phys pool index when materialised
    int spec = -1;       // work-spectrum index (band b2) when available
};

template <typename T>
class Engine : public EngineBase {
   public:
    explicit Engine(const mlq_params& p);
    ~Engine() override;

    // ---- buffers ----
    T* phys(int i);                       // N^3 physical scratch, lazily allocated (full mode)

    // ---- z-slab streaming (large N) ----
    // In slab mode no N^3 field is kept: a physical field index ("slot") is
    // backed by its pruned y-stage array (the output of the z stage, exact for
    // a band-limited field), by a pointwise recipe (a power of another slot),
    // by the constant 1, or, for host transfers, by a full buffer.  A forward
    // pipeline expands its inputs a slab of zs_ planes at a time through the
    // y/x inverse passes, runs the fused x stage and the y pass per slab, and
    // the z stages on whole arrays.
    bool slab_ = false;
    int zs_ = 0;  // planes per slab
    struct PSlot {
        enum Kind { NONE = 0, FULL, YS, RAW, ONE } kind = NONE;
        Band band{};      // YS: band of the stored y-stage array
        int src = -1;     // RAW: source slot
        double pk = 0.0;  // RAW: FGPow exponent and threshold flag
        int pthresh = 0;
    };
    std::vector<PSlot> slot_;
    std::vector<cpx<T>*> slot_ys_;  // YS storage, n * nbcap * nxcap
    std::vector<cpx<T>*> slot_pool_;  // released YS storage blocks, reused before allocating
    void release_slots(int lo, int hi);  // slots [lo, hi) no longer hold values
    PSlot& slot(int i);
    cpx<T>* slot_ys(int i);         // storage of slot i, allocated on first use
    std::vector<T*> slab_bufs_;     // zs_ * n^2 each
    std::vector<cpx<T>*> xslab_;    // zs_ * n * nxcap each
    T* slab_buf(int k);
    cpx<T>* xslab(int k);
    // physical values of slot i on planes [z0, z0 + zs_) into slab buffer k
    const T* expand(int i, int z0, int k);
    // physical values of several slots on planes [z0, z0 + zs_): slot in[k]
    // lands in slab buffer k; y-stage slots of one band share launches
    std::vector<const T*> expand_many(const std::vector<int>& in, int z0);
    bool ls_fits();  // room for the line-search setup's fields in slab mode
    void release_io_buffers();      // drop lazily allocated work buffers (state and twiddles stay)
    cpx<T>* xsbuf(int i);                 // [n][n][nxcap]
    cpx<T>* ysbuf(int i);                 // [n][nbcap][nxcap]
    cpx<T>* wspec(int i);                 // work spectrum in band b2, nb*nb*nx
    int nxcap, nbcap;
    // Row pitch (elements) of the x- and y-stage arrays of band b: rounded up
    // to even in FP32 with the compile-time kernels, so that every row starts
    // on a 16-byte boundary and two neighbouring kx columns move as one
    // 16-byte vector; the pad column is kept zero.  Spectra keep pitch nx.
    bool pitch_even_ = false;
    int px_of(int nx) const { return pitch_even_ ? ((nx + 1) & ~1) : nx; }
    int px_of(const Band& b) const { return px_of(b.nx); }
    int pxcap() const { return px_of(nxcap); }
    std::vector<T*> phys_;
    std::vector<cpx<T>*> xs_, ys_, ws_;

    // ---- pipelines ----
    struct FwdOut {
        void* spec = nullptr;
        int spec_f64 = 0;
        int phys_out = -1;   // round trip destination (phys index), -1 none
        int sym = SYM_ONE, ab = 0;
        const void* add = nullptr;
        int add_f64 = 0, add_sym = SYM_ONE, add_ab = 0;
        double add_coef = 0;
        int red_self = -1;
        const void* red_with[3] = {nullptr, nullptr, nullptr};
        int red_with_f64[3] = {0, 0, 0}, red_with_slot[3] = {-1, -1, -1};
    };
    // Forward pipeline of functor outputs through band b; reductions of the
    // z stage land in results[red_dst + slot] (slot < MAX_RED); functor
    // reductions in results[fred_dst + r].
    template <class F>
    void fwd(const Band& b, const F& f, const std::vector<int>& in, std::vector<FwdOut> outs, int red_dst = -1,
             int fred_dst = -1, double norm = -1.0);
    struct InvOut {
        ZSrc src[3];
        int nsrc = 0;
        int phys_out = -1;
    };
    void inv(const Band& b, const std::vector<InvOut>& outs);
    template <int NOUT>
    void fwd_z(const Band& b, const std::vector<FwdOut>& outs, int red_dst, double norm);
    template <class F>
    void fwd_slab(const Band& b, const F& f, const std::vector<int>& in, std::vector<FwdOut>& outs, int red_dst,
                  int fred_dst, double norm);
    template <class F>
    void pointwise(const F& f, const std::vector<int>& in, const std::vector<int>& out, int fred_dst = -1);
    void yx_inverse(const Band& b, const std::vector<cpx<T>*>& ys, const std::vector<int>& phys_out);

    // ---- programs ----
    // R parts at phi = u + tau*d (d may be null) -> results; also ||phi||_q^q.
    void R_eval(const SVec* u, const SVec* d, double tau, double out[3], double* lqq);
    // calc_global_dEnstrophydt (function_ops.f90:1417-1481): out = {R1 + R2, R1, R2}
    void dEnstrophydt(const SVec* u, double out[3]);
    // calc_local_pointwise_dLqdt_inclParts (1224-1291): the fields R1 + R2 +
    // R3, R1 + R2, R3 into the host (n,n,n,3) array
    void pointwise_R(const SVec* u, double* host);
    // L2 gradient of R at u (GradL2ForLq) into v (FP64 spectra); also the
    // dealiased |u|^{q-2} u spectra (for calcConstraintDerivativeL2) into
    // c (FP64, may be null) and ||u||_q^q.
    void grad_l2(const SVec* u, SVec* v, SVec* c, double* lqq);
    void grad_l2_body(const SVec* u, SVec* v, SVec* c, bool want_lq, bool from_retraction);
    int grad_lq_slot_ = 0;
    // vectorTransport pieces at w = u + tau*d: ir[i] = <P2(|w|^{q-2} w), xi_i>,
    // returns ||w||_q^q.
    double transport_pieces(const SVec* u, const SVec* d, double tau, const SVec* const* xi, int nxi,
                            double* ir);
    double lq_pow(const SVec* u, const SVec* d, double tau);  // ||u + tau d||_q^q
    // |u|^k physical (calc_uk) of the state u, into phys index dst
    void calc_uk(const SVec* u, double k, int dst);

    // Line search along phi = u + tau d when q = 4 (|u|^{q-4} = 1): the
    // setup forms the tau-coefficient fields once; a trial is then one
    // forward transform of g(tau)^2 plus polynomial evaluations.
    bool ls_ok() const { return !use_e_u && P.q == 4.0; }
    // tau0: the previous step, whose neighbourhood the trials visit (<= 0: none)
    void ls_setup(const SVec* u, const SVec* d, double tau0 = 0.0);
    void ls_trial(double tau, double out[3], double* lqq);
    // Where S(tau) = S0 + tau S1 + tau^2 S2 (the dealiased |phi|^2) is >= 0 at
    // every point, the clamp of calc_uk is inactive and P2(g^2) = S(tau): a
    // trial in [ls_c_.tlo, ls_c_.thi] is then a polynomial in tau of the
    // Parseval products <S_i, X_a> (X_a: coefficients of P2|grad phi|^2) and
    // <S_i, S_j>.
    LsPoly ls_c_{};
    bool ls_host_poly_ = true;  // ls_c_ holds this line search's coefficients
    void ls_poly_to_host();     // copies them from the device search's state
    long long ls_poly_trials_ = 0, ls_fft_trials_ = 0;

    // ---- the line search on the device ----
    // The setup leaves the coefficients in d_ls_ only (ls_dev_), and the
    // search runs as one CUDA graph: a conditional loop around the controller
    // kernel, which replays mnbrak and Brent over the trial values found so
    // far and stops at the first tau it has none for; inside the loop a
    // conditional check of S(tau) >= 0 at that tau and, where it fails, a
    // conditional transform trial.  The host reads the outcome once.
    // MLQ_DEVICE_LS=0 keeps the search on the host.
    bool ls_dev_on_ = true;
    // MLQ_LS_TRANSFORM_TRIALS=1: every trial by a transform, on host and
    // device alike (the polynomial shortcut off; for tests of that branch)
    bool ls_transform_trials_ = false;
    bool ls_dev_ = false;
    LsDevState* d_ls_ = nullptr;
    void* h_ls_ = nullptr;  // pinned: LsParams, LsOut, LsPoly
    struct LsGraph {
        cudaGraphExec_t exec = nullptr;
        long gen = -1;
        int key = -1;
        long long nfwd = 0;  // launches of one transform trial
    };
    LsGraph lsg_[2];
    bool lsg_failed_ = false;
    long long ls_dev_searches_ = 0, ls_dev_loops_ = 0;
    double ls_free_tau_ = 0.0;  // the last device search's tau1 and whether
    int ls_free_val_ = -1;      // S(tau1) >= 0 everywhere (-1: none)
    bool ls_device_ready() const { return ls_dev_on_ && graphs_on_ && !slab_ && !lsg_failed_; }
    // 0: the search ran (out filled); 1: not available, search on the host
    int ls_device_search(double B, double tA0, double tB0, LsOut* out);
    bool ls_graph_build(LsGraph& g, int key);

    // ---- state <-> host ----
    // Forward transform of a host FP64 vector field into state spectra.
    // Returns the relative energy outside the band.
    // spec_f64: storage of spec (-1: this engine's state storage)
    double load_vec(const double* host, SVec* spec, int spec_f64 = -1);
    void store_vec(const SVec* spec, double* host, int spec_f64 = -1);
    // xs: a copy stream to run on instead of the engine's (not in slab mode);
    // both return when their copies are done
    void load_scalar_phys(const double* host, int dst, cudaStream_t xs = nullptr);
    void store_scalar_phys(int src, double* host, cudaStream_t xs = nullptr);
    cudaStream_t xstream_ = nullptr;
    cudaStream_t copy_stream();

    // ---- full-band FFT API (fftwfunction.f90) ----
    void fft_c2c(const double* in, double* out, int sign);
    void fft_r2c(const double* in, double* out);
    void fft_c2r(const double* in, double* out);
    void dealias_scalar(double* g, double order);
    // function_ops.f90 operators on arbitrary (not band-limited) fields, in
    // the full band: gradient (3147), divergence (3200), laplacian (3248),
    // solve_poisson (1951)
    void gradient_full(const double* f, double* grad);
    void divergence_full(const double* u, double* div);
    void laplacian_full(double* u);
    void poisson_full(const double* f, double l, double* phi);
    // kappa_test_pert (function_ops.f90:615-977): the gradient-check
    // perturbations, full band; returns 0, or 1 for a load-* type without
    // its field (formed from zeros: the reference's successful = .false.)
    int kappa_pert(const char* type, double m1, double m2, double m3, const double* loaded, unsigned long long seed,
                   double* out);
    void widen_to(const Band& b);

    SVec* c_tmp_ = nullptr;  // FP64 spectra of P2(|w|^{q-2} w) for the transport
    double* d_coef_ = nullptr;  // cs, tau of the retraction (read by a captured launch)
    void phys_written(int idx);  // clears the physical-field memo when it covers idx
    bool w_from_memo(const SVec* u, const SVec* d, double tau);
    bool ls_clamp_free(double tau);  // S(tau) >= 0 at every point (the interval, else one check)
    int ls_p0_ = -1, ls_w0_ = -1;    // physical field and work spectrum of S_0 in this line search
    int ls_phys(int a) const;        // physical field of S_a
    int ls_wspec(int a) const;       // work spectrum of S_a

    // register-resident FFT kernels (power-of-two n >= 64); E elements per thread
    int ereg_ = 8;  // elements per thread: 8 up to n = 512, 16 above
    bool reg_ok_ = false;
    cpx<T>* d_twT_ = nullptr;  // twiddle pool in T
    RPlan rplan(int L) const;
    // kernels specialised at compile time for n in {64, ..., 1024} (cfft.cuh)
    bool cfft_ok_ = false;
    int persistent_blocks(const void* kernel, int threads, size_t smem);
    std::map<const void*, int> occ_;
    int num_sms_ = 148;
    template <int NN>
    void xinv_c(XInvArgs<T>& xa, int narr);
    template <int NN, class F>
    void xfwd_c(XFwdArgs<T>& xa, const F& f);
    long last_xblocks_ = 0;  // reduction records of the last x-stage launch
    template <int NN>
    void y_c(YArgs<T>& ya, int sign, int narr);
    template <int NN, int V>
    void y_cv(YArgs<T>& ya, int sign, int narr);
    template <int NN, int V>
    void zfwd_cv(ZFwdArgs<T>& za, int narr);
    template <int NN, int V>
    void zinv_cv(ZInvArgs<T>& za, int narr);
    template <int NN, int V>
    void zinv_multi_cv(ZInvMultiArgs<T>& za, int nops);
    // z inverse of ops that each share one source among up to ZMULTI outputs
    void launch_zinv_multi(ZInvMultiArgs<T>& za, int nops, const Band& b, double zbytes);
    template <int NN, class Fn>
    void with_variant(int kind, Fn&& f);
    // y/z tile-shape variant per pass kind, chosen by tune_yz()
    // (YV_ZRT: z forward launches with a round trip back into the y stage)
    enum { YV_YFWD = 0, YV_YINV = 1, YV_ZFWD = 2, YV_ZINV = 3, YV_ZRT = 4, YV_KINDS = 5 };
    int yvar_[YV_KINDS] = {0, 0, 0, 0, 0};
    void tune_yz();
    std::string tune_report_;
    std::string kernel_config() const override;
    template <int NN>
    void zfwd_c(ZFwdArgs<T>& za, int narr);
    template <int NN>
    void zinv_c(ZInvArgs<T>& za, int narr);
    int reg_tx() const;
    int reg_lx(int nrows_per_line, size_t pitch) const;
    // pass launchers (register kernels when reg_ok_, shared-memory Stockham otherwise)
    template <class F>
    void launch_xfwd(XFwdArgs<T>& xa, const F& f, int nout, const Band& b);
    void launch_y(YArgs<T>& ya, int sign, int narr, const Band& b);
    void launch_zfwd(ZFwdArgs<T>& za, int narr, const Band& b, bool any_rt, double zbytes);
    void launch_zinv(ZInvArgs<T>& za, int narr, const Band& b, double zbytes);
    void launch_xinv(XInvArgs<T>& xa, int narr, const Band& b);
    long last_zblocks_ = 0;

   private:
    // |u|^k chain (calc_uk); memoised per program
    std::map<double, PowField> memo_;
    int tmp_next_ = 0, spec_next_ = 0;
    void chain_reset() {
        memo_.clear();
        tmp_next_ = 0;
        spec_next_ = 0;
    }
    PowField chain(double k);
    void ensure_p2_spec(PowField& f);
    void ensure_phys(PowField& f);
    cpx<T>* ones_spec();
    void A_and_S(bool need_A_phys);
    int lx_for(int nout, size_t extra = 0) const;
    int tx_for() const;
    double* h_stage_ = nullptr;  // pinned staging for host copies
    size_t h_stage_bytes_ = 0;
    void* stage(size_t bytes);
};

}  // namespace mlq
