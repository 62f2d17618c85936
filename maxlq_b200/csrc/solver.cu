// solver.cu -- the CG search (optimization.f90) on the engine.
#include "solver.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <type_traits>
#include <vector>

namespace mlq {

void seed_spectrum_host(int n, unsigned long long seed, double slope, double k0, const Band& b, double* out);

namespace {
const double TAU_MAX = 1.0e2;  // global_variables.f90:29
std::string fmt_e(double v) {
    char b[32];
    snprintf(b, sizeof(b), "%.3e", v);
    return b;
}
}  // namespace

template <typename T>
class Solver : public SolverBase {
   public:
    Engine<T> e;
    SVec *u, *d1, *gu0, *gu1, *vtg0, *vtd0, *c, *tmp, *tmp2;
    // CG memory of the resident loop
    bool started = false;
    int iter = 0, start_iter = 0;
    double J0 = 0, tau0 = 100.0;
    std::vector<double> roll;
    double avg_imp = 1.0;
    int while_flag = 0;
    std::map<double, Trial> trials;

    // Host transfers of FP64 state always go through an FP64 pipeline, so a
    // stored field is the exact field of the FP64 state spectra in both modes.
    std::unique_ptr<Engine<double>> io64_;
    Engine<double>& io() {
        if constexpr (std::is_same<T, double>::value) {
            return e;
        } else {
            if (!io64_) io64_.reset(new Engine<double>(e.P));
            return *io64_;
        }
    }

    // In slab mode memory is tight: the FP64 transfer pipeline of a mixed
    // context gives its work buffers back after each host transfer.
    void trim_io() {
        if (e.slab_ && io64_) io64_->release_io_buffers();
    }

    explicit Solver(const mlq_params& p) : e(p) {
        u = e.alloc_state();
        d1 = e.alloc_state();
        gu0 = e.alloc_state();
        gu1 = e.alloc_state();
        vtg0 = e.alloc_state();
        vtd0 = e.alloc_state();
        c = e.alloc_state();
        tmp = e.alloc_state();
        tmp2 = nullptr;
    }
    EngineBase& eng() override { return e; }
    long nc() const { return e.spec_ncomp(); }
    double q() const { return e.P.q; }
    double B() const { return e.P.B; }

    void zero(SVec* f) { MLQ_CUDA(cudaMemsetAsync(f, 0, 3 * nc() * e.sv_elem(), e.stream)); }

    // load a host vector field, refusing fields with modes outside the band
    void load(const double* host, SVec* spec) {
        MLQ_CUDA(cudaStreamSynchronize(e.stream));
        e.state_written(spec);
        const double rel = io().load_vec(host, spec, e.sf64());
        trim_io();
        const double tol = 1e-24;  // relative energy; FP64 FFT round-trip noise is ~1e-32
        if (std::isnan(rel))
            throw CudaError("input field holds NaN or Inf (the reference stops at fftwfunction.f90:78-89)",
                            MLQ_ERR_NAN);
        if (!(rel <= tol))
            throw CudaError("input field is not band-limited to the 2/3 dealiasing cube (relative energy outside: " +
                                fmt_e(rel) + ")",
                            MLQ_ERR_NOT_BANDLIMITED);
    }

    // ---- line search -------------------------------------------------------
    // Line-search trials go through the polynomial path when q = 4: setup
    // once per (base, dir), then one transform per trial.
    bool ls_ready = false;
    // tau_near: a step the trials will visit the neighbourhood of (the
    // previous step in the CG loop), for the setup's clamp-free intervals
    void ls_begin(const SVec* base, const SVec* dir, double tau_near = 0.0) {
        trials.clear();
        ls_ready = false;
        if (e.ls_ok() && dir && e.ls_fits()) {
            e.ls_setup(base, dir, tau_near);
            ls_ready = true;
        }
    }
    Trial trial(const SVec* base, const SVec* dir, double tau) {
        auto it = trials.find(tau);
        if (it != trials.end()) return it->second;
        Trial t;
        if (ls_ready)
            e.ls_trial(tau, t.R, &t.lqq);
        else
            e.R_eval(base, dir, tau, t.R, &t.lqq);
        trials[tau] = t;
        return t;
    }
    // eval_J(phi + tau d, "LineMin") (optimization.f90:537-539)
    double lm_eval(const SVec* base, const SVec* dir, double tau) {
        ++eval_count;
        ++evals_this_iter;
        const Trial t = trial(base, dir, tau);
        const double J = ls_J(t.R[1], t.R[2], t.lqq, q(), B());
        // The reference's trial rescales the field and transforms it; a NaN
        // there stops the program at the FFT's NaN scan (fftwfunction.f90:78-89).
        // A trial that needs no transform (homogeneity, polynomial path)
        // reports the same condition from its value.
        if (std::isnan(J)) throw CudaError("NaN in a line-search trial value", MLQ_ERR_NAN);
        return J;
    }
    double scaled_R(const Trial& t) const { return -ls_J(t.R[1], t.R[2], t.lqq, q(), B()); }
    int evals_this_iter = 0;

    // the host evaluator of the line-search templates (linesearch.cuh)
    struct HostEval {
        Solver* s;
        const SVec* phi;
        const SVec* dir;
        bool operator()(double tau, double* J) {
            *J = s->lm_eval(phi, dir, tau);
            return true;
        }
    };
    // mnbrak (optimization.f90:613-778)
    int mnbrak(const SVec* phi, const SVec* grad, double tA0, double tB0, double tau_brack[2], int* myflag) {
        HostEval ev{this, phi, grad};
        return ls_mnbrak(ev, tA0, tB0, tau_brack, myflag);
    }
    // brent (optimization.f90:784-951)
    double brent(const SVec* phi, const SVec* grad, const double tau_brack[2], double* fx_out) {
        HostEval ev{this, phi, grad};
        double x = 0.0;
        ls_brent(ev, tau_brack, &x, fx_out);
        return x;
    }

    // ---- CG loop -------------------------------------------------------------
    double H(const SVec* a, const SVec* b) {
        SpecDotPair p{a, b, 1};
        double r;
        e.dots(&p, 1, &r);
        return r;
    }

    void pre_loop() {
        // rescaleLqNorm + divAvg_free (optimization.f90:61-62)
        const double nrm = std::pow(e.lq_pow(u, nullptr, 0.0), 1.0 / q());
        e.lincomb(u, B() / nrm, u);
        e.leray(u);
        Trial t;
        e.R_eval(u, nullptr, 0.0, t.R, &t.lqq);
        J0 = t.R[0];  // 78
        iter = start_iter;
        tau0 = std::pow(10.0, 2.0);
        zero(gu0);
        zero(vtg0);
        zero(vtd0);
        roll.assign(std::max(1, e.P.rolling_size), 0.0);
        avg_imp = 1.0;
        while_flag = 0;
        started = true;
    }

    // one iteration of optimization.f90:136-446; returns status
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    // device time of one iteration: CUDA events on the engine's stream
    void iter_clock_start() {
        if (!ev0_) {
            MLQ_CUDA(cudaEventCreate(&ev0_));
            MLQ_CUDA(cudaEventCreate(&ev1_));
        }
        MLQ_CUDA(cudaEventRecord(ev0_, e.stream));
    }
    double iter_clock_stop() {
        MLQ_CUDA(cudaEventRecord(ev1_, e.stream));
        MLQ_CUDA(cudaEventSynchronize(ev1_));
        float ms = 0.f;
        MLQ_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
        return ms * 1e-3;
    }

    int one_iteration(mlq_iter_info& info) {
        iter_clock_start();
        std::memset(&info, 0, sizeof(info));
        iter++;
        info.iter = iter;
        evals_this_iter = 0;
        trials.clear();
        const double qq = q(), Bc = B();
        const double s = (3.0 / 2.0) - (1.0 / qq);  // 150
        SVec* g1 = gu1;
        double lqq_u = 0;
        e.grad_l2(u, g1, c, &lqq_u);  // 146
        // Hilbert gradient of g (151, 153) and of the normal of the tangent
        // space ||u||_q^{1-q} P2(|u|^{q-2} u) (162, 164, 169), with <c, g>
        // and <c, c> (170-171) in the same pass
        const double unorm = std::pow(lqq_u, 1.0 / qq);
        double dd[2];
        e.hilbert_leray_pair_dots(g1, c, s, std::pow(unorm, 1.0 - qq), dd);
        const double alpha = dd[0] / dd[1];  // 170-171
        info.alpha = alpha;
        if (!e.P.use_tangential_gradient) throw CudaError("useTangentialGradient=.false. is not supported",
                                                          MLQ_ERR_BADARG);
        // Every inner product the rest of the update needs, in one pass.  The
        // reference forms g + c (180-193) and g - T g0 (223-226) and the norm
        // of d1 only to take inner products of them; those are expanded here
        // into products of g, c, u, T g0, g0, T d0 (bilinearity), which
        // saves two state-vector temporaries and four reductions.
        const double cc = dd[1];  // <c, c>
        enum { GC, GDIV, GG, UU, GTG, G0G0, GTD, TDTD };
        double ip[8];
        {
            // gradJproj g <- g - alpha c (177, kept in gu1) in the same pass
            SpecDotPair p[8] = {{g1, c, 1},    {g1, nullptr, 2}, {g1, g1, 1},   {u, u, 1},
                                {g1, vtg0, 1}, {gu0, gu0, 1},    {g1, vtd0, 1}, {vtd0, vtd0, 1}};
            e.dots(p, 8, ip, g1, g1, -alpha, c);
        }
        info.ortho_check = std::fabs(ip[GC] / (ip[GG] + 2.0 * ip[GC] + cc));  // <g,c> / <g+c, g+c>
        info.div_check = ip[GDIV] / ip[GG];
        double sg = 1.0;  // gradient normalisation (213), applied with d1 below
        if (e.P.normalize_gradient) sg = std::sqrt(ip[UU] / ip[GG]);
        const double gg = sg * sg * ip[GG], gtd = sg * ip[GTD];  // <g', g'>, <g', T d0>
        double beta = 0.0;
        if (e.P.use_conjugate_gradient) {
            beta = gg - sg * ip[GTG];  // <g', g' - T g0> (226)
            const double g0n = ip[G0G0];  // 227
            if (g0n < MACH_EPSILON || beta < MACH_EPSILON)
                beta = 0.0;
            else
                beta = beta / g0n;
            if (e.P.reset_momentum_every > 0 && iter % e.P.reset_momentum_every == 0) beta = 0.0;  // 235-238
            e.direction(g1, sg, d1, beta, vtd0);                                                     // 213, 240
        } else {
            e.direction(g1, sg, d1, 0.0, nullptr);
        }
        info.beta = beta;
        info.norm_grad = std::sqrt(gg);
        info.norm_td0 = std::sqrt(ip[TDTD]);
        info.norm_d1 = std::sqrt(std::max(0.0, gg + 2.0 * beta * gtd + beta * beta * ip[TDTD]));
        e.zeroth(d1, info.mean_d1);  // 251
        e.zeroth(u, info.mean_u);    // 257
        // line search (269-318)
        double tb[2] = {0, 0};
        int mflag = 0;
        ls_begin(u, d1, tau0);
        double fx = 0, tau1 = 0;
        LsOut lo;
        if (ls_ready && e.ls_device_search(Bc, 0.0, tau0, &lo) == 0 && lo.status != LS_ERR_CAP) {
            // mnbrak and Brent ran on the device; one read of the outcome
            eval_count += lo.evals;
            evals_this_iter += lo.evals;
            if (lo.status == MLQ_ERR_NAN) throw CudaError("NaN in a line-search trial value", MLQ_ERR_NAN);
            mflag = lo.mflag;
            tb[0] = lo.tb[0];
            tb[1] = lo.tb[1];
            if (mflag == 0) {
                tau1 = lo.tau1;
                fx = lo.fx;
                Trial t;
                for (int k = 0; k < 3; ++k) t.R[k] = lo.R1[k];
                t.lqq = lo.lqq1;
                trials[tau1] = t;
            }
        } else {
            mnbrak(u, d1, 0.0, tau0, tb, &mflag);
            if (mflag == 0) tau1 = brent(u, d1, tb, &fx);  // 297
        }
        info.J0 = J0;
        info.mnbrak_flag = mflag;
        if (mflag != 0) {
            info.n_evals = evals_this_iter;
            info.status = mflag == 1 ? MLQ_ERR_MNBRAK_UPHILL : MLQ_ERR_MNBRAK_ITMAX;
            while_flag = 1;
            info.seconds = iter_clock_stop();
            return info.status;
        }
        info.tau_a = tb[0];
        info.tau_b = tb[1];
        int status = MLQ_OK;
        if (tau1 > TAU_MAX) {  // 310-314
            while_flag = 1;
            status = MLQ_ERR_TAU_MAX;
            tau1 = 0.0;
        }
        info.tau = tau1;
        // vector transport of gu1 and d1 to the new point (324-328)
        double ir[2];
        const SVec* xi[2] = {g1, d1};
        ls_ready = false;
        double lqw;
        if (e.P.use_riemannian_geometry)
            lqw = e.transport_pieces(u, d1, tau1, xi, 2, ir);
        else
            lqw = e.lq_pow(u, d1, tau1);
        const double ln = std::pow(lqw, 1.0 / qq);
        // R at the retracted point from the accepted trial (homogeneity), as
        // eval_J(Uvec, "maxdLqdt") after rescaleLqNorm (344-349)
        const Trial tr = trial(u, d1, tau1);
        const double cs = Bc / std::pow(tr.lqq, 1.0 / qq);
        const double R12n = std::pow(cs, qq) * tr.R[1], R3n = std::pow(cs, qq + 1.0) * tr.R[2];
        if (e.P.use_riemannian_geometry) {
            // transported gradient and direction (324-328), then u <- (B/ln) w
            const double f = std::pow(ln, -qq);
            e.transport_retract(vtg0, vtd0, g1, d1, u, Bc / ln, -Bc / ln * f * ir[0], -Bc / ln * f * ir[0] * tau1,
                                Bc / ln, -Bc / ln * f * ir[1], -Bc / ln * f * ir[1] * tau1, Bc / ln, tau1);
        } else {
            e.lincomb(vtg0, 1.0, g1);
            e.lincomb(vtd0, 1.0, d1);
            e.retract(u, Bc / ln, tau1, d1);
        }
        trials.clear();
        const double J1 = R12n + R3n;
        const double deltaJ = (J1 - J0) / std::fabs(J0);
        info.J1 = J1;
        info.deltaJ = deltaJ;
        info.n_evals = evals_this_iter;
        if (deltaJ < -MACH_EPSILON) {  // 351-366
            while_flag = 1;
            info.status = MLQ_ERR_J_DECREASED;
            info.seconds = iter_clock_stop();
            return info.status;
        }
        info.u_norm_q = cs * std::pow(tr.lqq, 1.0 / qq);  // ||u||_q after the retraction (421)
        info.R = J1;
        info.R12 = R12n;
        info.R3 = R3n;
        // 432-445
        J0 = J1;
        std::swap(gu0, gu1);
        tau0 = tau1;
        for (int i = (int)roll.size() - 1; i >= 1; --i) roll[i] = roll[i - 1];
        roll[0] = deltaJ;
        double ssum = 0.0;
        for (double r : roll) ssum += r;
        avg_imp = ssum / (double)(iter - start_iter);
        info.status = status;
        info.seconds = iter_clock_stop();
        return status;
    }

    int state_iterate(int n_iter, mlq_iter_cb cb, void* user, int* iters) override {
        if (!started) pre_loop();
        int done = 0, status = MLQ_OK;
        while (done < n_iter && std::fabs(avg_imp) > e.P.optim_tol && iter < e.P.max_iter && while_flag < 1) {
            mlq_iter_info info;
            status = one_iteration(info);
            ++done;
            if (cb) cb(&info, user);
            if (status != MLQ_OK) break;
        }
        if (iters) *iters = iter;
        return status;
    }

    // ---- host-array entry points ----------------------------------------------
    void R_parts(const double* uh, double out[3]) override {
        load(uh, tmp);
        double lqq;
        e.R_eval(tmp, nullptr, 0.0, out, &lqq);
    }
    double eval_J(const double* uh, int mode) override {
        load(uh, tmp);
        Trial t;
        switch (mode) {
            case MLQ_J_MAXDLQDT:
                e.R_eval(tmp, nullptr, 0.0, t.R, &t.lqq);
                return t.R[0];
            case MLQ_J_LINEMIN:
                ++eval_count;
                e.R_eval(tmp, nullptr, 0.0, t.R, &t.lqq);
                return -1.0 * scaled_R(t);
            case MLQ_J_LQNORM:
                return std::pow(e.lq_pow(tmp, nullptr, 0.0), 1.0 / q());
        }
        throw CudaError("unknown eval_J mode", MLQ_ERR_BADARG);
    }
    void grad_l2(const double* uh, double* v) override {
        load(uh, tmp);
        e.grad_l2(tmp, d1, c, nullptr);
        store(d1, v);
        started = false;
    }
    double lq_norm(const double* uh) override {
        load(uh, tmp);
        return std::pow(e.lq_pow(tmp, nullptr, 0.0), 1.0 / q());
    }
    void rescale(double* uh, double Bv) override {
        const double nrm = lq_norm(uh);
        const long m = 3 * e.n3;
        for (long i = 0; i < m; ++i) uh[i] = Bv / nrm * uh[i];
    }
    void normal_l2(const double* uh, double* out) override {
        load(uh, tmp);
        // |u|^{q-2}u dealiased (984-1006): the same spectra grad_l2 builds
        double lqq;
        e.grad_l2(tmp, d1, c, &lqq);
        const double nrm = std::pow(lqq, 1.0 / q());
        e.lincomb(c, std::pow(nrm, 1.0 - q()), c);
        store(c, out);
        started = false;
    }
    void vector_transport(const double* uh, double qv, double Bv, const double* eta, const double* xi,
                          double* out) override {
        if (qv != q()) throw CudaError("vectorTransport q must equal the context's q", MLQ_ERR_BADARG);
        load(uh, tmp);
        load(eta, d1);
        load(xi, gu1);
        double ir;
        const SVec* xs[1] = {gu1};
        const double lqq = e.transport_pieces(tmp, d1, 1.0, xs, 1, &ir);
        const double ln = std::pow(lqq, 1.0 / qv);
        const double f = std::pow(ln, -qv) * ir;
        e.lincomb(c, Bv / ln, gu1, -Bv / ln * f, tmp, -Bv / ln * f, d1);
        store(c, out);
        started = false;
    }
    void hilbert_host(double* g, double order) override {
        load(g, tmp);
        e.hilbert(tmp, order);
        store(tmp, g);
    }
    void divavg_host(double* g) override {
        load(g, tmp);
        e.leray(tmp);
        store(tmp, g);
    }
    double inner_host(const double* f, const double* g, int type) override {
        load(f, tmp);
        load(g, c);
        SpecDotPair p{tmp, c, type == MLQ_INNER_HL ? 1 : 0};
        double r;
        e.dots(&p, 1, &r);
        started = false;
        return r;
    }
    void zeroth_host(const double* uh, double out[3]) override {
        load(uh, tmp);
        e.zeroth(tmp, out);
    }
    void calc_uk_host(const double* uh, double k, double* out) override {
        load(uh, tmp);
        e.calc_uk(tmp, k, 40);
        e.store_scalar_phys(40, out);
    }
    void spectral_data_host(const double* uh, int normalize, double* out) override {
        load(uh, tmp);
        e.spectrum(tmp, normalize != 0, out);
    }
    void state_spectral_data(int normalize, double* out) override { e.spectrum(u, normalize != 0, out); }
    double enstrophy_host(const double* uh) override {
        load(uh, tmp);
        return e.enstrophy(tmp);
    }
    void dEnstrophydt_host(const double* uh, double out[3]) override {
        load(uh, tmp);
        e.dEnstrophydt(tmp, out);
    }
    void pointwise_R_host(const double* uh, double* out) override {
        load(uh, tmp);
        e.pointwise_R(tmp, out);
    }
    int mnbrak_host(const double* phi, const double* d, double tA0, double tB0, double br[2], int* flag) override {
        load(phi, tmp);
        load(d, c);
        ls_begin(tmp, c, tB0);
        *flag = 0;
        mnbrak(tmp, c, tA0, tB0, br, flag);
        trials.clear();
        started = false;
        return *flag;
    }
    double brent_host(const double* phi, const double* d, const double br[2]) override {
        load(phi, tmp);
        load(d, c);
        ls_begin(tmp, c, std::max(br[0], br[1]) * 0.381966);
        const double x = brent(tmp, c, br, nullptr);
        trials.clear();
        started = false;
        return x;
    }
    void state_load(const double* uh) override {
        load(uh, u);
        started = false;
    }
    void store(const SVec* spec, double* host) {
        MLQ_CUDA(cudaStreamSynchronize(e.stream));
        io().store_vec(spec, host, e.sf64());
        trim_io();
    }
    void state_store(double* uh) override { store(u, uh); }
    int state_step(double* uh, mlq_iter_cb cb, void* user) override {
        load(uh, u);  // CG memory (gu0, vtg0, vtd0, tau0, J0, rolling average) kept
        int it = 0;
        const int st = state_iterate(1, cb, user, &it);
        store(u, uh);
        return st;
    }
    void state_R(double out[3], double* lqn) override {
        double lqq;
        e.R_eval(u, nullptr, 0.0, out, &lqq);
        if (lqn) *lqn = std::pow(lqq, 1.0 / q());
    }
    void seed_field(unsigned long long seed, double slope, double k0, double* out) override {
        std::vector<double> h(3 * nc() * 2);
        seed_spectrum_host(e.n, seed, slope, k0, e.b2, h.data());
        // through an FP64 buffer of the FP64 transfer engine: the seeded field
        // exactly, whatever the state storage of this context
        Engine<double>& io64 = io();
        SVec* t = io64.dev_alloc(3 * nc() * sizeof(double2));
        MLQ_CUDA(cudaMemcpyAsync(t, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, io64.stream));
        io64.store_vec(t, out, 1);
        io64.free_dev(t);
        trim_io();
    }
    void set_B(double Bv) override {
        e.P.B = Bv;
        started = false;
    }
    void set_start_iter(int s) override { start_iter = s; }
};

std::unique_ptr<SolverBase> make_solver(const mlq_params& p) {
    if (p.precision == MLQ_PREC_MIXED) return std::unique_ptr<SolverBase>(new Solver<float>(p));
    return std::unique_ptr<SolverBase>(new Solver<double>(p));
}

std::unique_ptr<EngineBase> make_fft_engine(const mlq_params& p) {
    mlq_params q = p;
    q.precision = MLQ_PREC_FP64;
    return std::unique_ptr<EngineBase>(new Engine<double>(q));
}

}  // namespace mlq
