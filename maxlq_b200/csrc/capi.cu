// capi.cu -- extern "C" entry points of libmaxlq_b200.so (include/maxlq.h).
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "solver.cuh"

using namespace mlq;

struct mlq_ctx {
    mlq_params p;
    std::unique_ptr<SolverBase> solver;
    std::unique_ptr<EngineBase> fft;  // FP64 engine for the fftwfunction API
    std::string err;
};

namespace mlq {
int band_cut_for_order(int n, double order);

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): a counter-based generator, so every Fourier mode draws
// its own numbers independently of the grid size and of the order of work.
// ---------------------------------------------------------------------------
static inline void philox_round(uint32_t ctr[4], const uint32_t key[2]) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t c0 = hi1 ^ ctr[1] ^ key[0];
    const uint32_t c2 = hi0 ^ ctr[3] ^ key[1];
    ctr[0] = c0;
    ctr[1] = lo1;
    ctr[2] = c2;
    ctr[3] = lo0;
}
void philox4x32_10(const uint32_t in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t ctr[4] = {in[0], in[1], in[2], in[3]};
    uint32_t key[2] = {key_in[0], key_in[1]};
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            key[0] += 0x9E3779B9u;
            key[1] += 0xBB67AE85u;
        }
        philox_round(ctr, key);
    }
    std::memcpy(out, ctr, sizeof(ctr));
}

// Two standard normals for mode (jx, jy, jz) and component c (Box-Muller on
// two 53-bit uniforms in (0,1)).
static void mode_normals(unsigned long long seed, int jx, int jy, int jz, int c, double* a, double* b) {
    const uint32_t key[2] = {(uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32)};
    const uint32_t ctr[4] = {(uint32_t)jx, (uint32_t)jy, (uint32_t)jz, (uint32_t)c};
    uint32_t r[4];
    philox4x32_10(ctr, key, r);
    const uint64_t m1 = (((uint64_t)r[0] << 32) | r[1]) >> 11;
    const uint64_t m2 = (((uint64_t)r[2] << 32) | r[3]) >> 11;
    const double u1 = ((double)m1 + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = ((double)m2 + 0.5) * (1.0 / 9007199254740992.0);
    const double rr = std::sqrt(-2.0 * std::log(u1));
    const double th = 2.0 * 3.14159265358979323846 * u2;
    *a = rr * std::cos(th);
    *b = rr * std::sin(th);
}

// Pruned half spectrum of a seeded, divergence-free, mean-free field in band
// b: u_hat(j) = A(|j|) (a + i b)/sqrt(2), A = |j|^-slope exp(-(|j|/k0)^2),
// Hermitian on the jx = 0 plane, then Leray-projected.  Layout [3][nb][nb][nx]
// complex (compact index order 0..cut, -cut..-1).
void seed_spectrum_host(int n, unsigned long long seed, double slope, double k0, const Band& b, double* out) {
    const long nc = (long)b.nb * b.nb * b.nx;
    std::memset(out, 0, sizeof(double) * 2 * 3 * nc);
    auto sj = [&](int ci) { return ci <= b.cut ? ci : ci - b.nb; };
    for (int cz = 0; cz < b.nb; ++cz)
        for (int cy = 0; cy < b.nb; ++cy)
            for (int cx = 0; cx < b.nx; ++cx) {
                const int jx = cx, jy = sj(cy), jz = sj(cz);
                if (jx == 0 && jy == 0 && jz == 0) continue;
                // canonical representative on the jx = 0 plane
                bool conj = false;
                int gy = jy, gz = jz;
                if (jx == 0 && (jy < 0 || (jy == 0 && jz < 0))) {
                    conj = true;
                    gy = -jy;
                    gz = -jz;
                }
                const double kk = std::sqrt((double)jx * jx + (double)jy * jy + (double)jz * jz);
                const double amp = std::pow(kk, -slope) * std::exp(-(kk / k0) * (kk / k0)) / std::sqrt(2.0);
                double re[3], im[3];
                for (int c = 0; c < 3; ++c) {
                    double a, bb;
                    mode_normals(seed, jx, gy, gz, c, &a, &bb);
                    re[c] = amp * a;
                    im[c] = conj ? -amp * bb : amp * bb;
                }
                // Leray projection with the integer wavevector
                const double jv[3] = {(double)jx, (double)jy, (double)jz};
                const double j2 = kk * kk;
                const double dr = (jv[0] * re[0] + jv[1] * re[1] + jv[2] * re[2]) / j2;
                const double di = (jv[0] * im[0] + jv[1] * im[1] + jv[2] * im[2]) / j2;
                const long idx = ((long)cz * b.nb + cy) * b.nx + cx;
                for (int c = 0; c < 3; ++c) {
                    out[2 * (c * nc + idx)] = re[c] - jv[c] * dr;
                    out[2 * (c * nc + idx) + 1] = im[c] - jv[c] * di;
                }
            }
}
}  // namespace mlq

namespace {
template <class Fn>
int guard(mlq_ctx* c, Fn fn) {
    if (!c) return MLQ_ERR_BADARG;
    try {
        fn();
        c->err.clear();
        return MLQ_OK;
    } catch (const CudaError& e) {
        c->err = e.what();
        return e.status;
    } catch (const std::exception& e) {
        c->err = e.what();
        return MLQ_ERR_CUDA;
    }
}
EngineBase& fft_engine(mlq_ctx* c) {
    if (!c->fft) c->fft = make_fft_engine(c->p);
    return *c->fft;
}
Engine<double>& fft64(mlq_ctx* c) { return static_cast<Engine<double>&>(fft_engine(c)); }
}  // namespace

extern "C" {

void mlq_default_params(mlq_params* p, int n, double q, double B) {
    std::memset(p, 0, sizeof(*p));
    p->n = n;
    p->q = q;
    p->B = B;
    p->visc = 1.0;
    p->lambda1 = 0.1;
    p->visc_coef = 1.0;
    p->press_coef = 1.0;
    p->to_dealias = 1;
    p->use_e_u_auto = 1;
    p->use_e_u = 1;
    p->dealias_e_u = 1;
    p->use_tangential_gradient = 1;
    p->use_conjugate_gradient = 1;
    p->use_riemannian_geometry = 1;
    p->normalize_gradient = 1;
    p->reset_momentum_every = 25;
    p->rolling_size = 10;
    p->max_iter = 99999;
    p->optim_tol = n >= 1024 ? 1.0e-4 : 1.0e-5;  // setStandardParams (initialize.f90:96-100)
    p->precision = MLQ_PREC_FP64;
    p->device = 0;
}

int mlq_init(mlq_ctx** out, const mlq_params* p) {
    if (!out || !p) return MLQ_ERR_BADARG;
    *out = nullptr;
    std::unique_ptr<mlq_ctx> c(new mlq_ctx);
    c->p = *p;
    int st = guard(c.get(), [&] { c->solver = make_solver(*p); });
    if (st != MLQ_OK) {
        // report through stderr: there is no context to query
        fprintf(stderr, "mlq_init: %s\n", c->err.c_str());
        return st;
    }
    *out = c.release();
    return MLQ_OK;
}

int mlq_finalize(mlq_ctx* c) {
    if (!c) return MLQ_ERR_BADARG;
    c->solver.reset();
    c->fft.reset();
    delete c;
    return MLQ_OK;
}

const char* mlq_last_error(const mlq_ctx* c) { return c ? c->err.c_str() : "null context"; }

int mlq_set_B(mlq_ctx* c, double B) {
    return guard(c, [&] {
        c->p.B = B;
        c->solver->set_B(B);
    });
}

long long mlq_kernel_launches(const mlq_ctx* c) {
    if (!c) return 0;
    long long k = c->solver ? c->solver->eng().launches : 0;
    if (c->fft) k += c->fft->launches;
    return k;
}

long long mlq_device_bytes(const mlq_ctx* c) {
    if (!c) return 0;
    long long b = c->solver ? c->solver->eng().bytes : 0;
    if (c->fft) b += c->fft->bytes;
    return b;
}

// fftfwd's NaN scan (fftwfunction.f90:78-89): a NaN in the real part of an
// output stops the reference; here the call returns MLQ_ERR_NAN.
static void nan_scan_real_parts(const double* fu, long n3) {
    for (long i = 0; i < n3; ++i)
        if (std::isnan(fu[2 * i])) throw CudaError("NaN in the forward transform's output", MLQ_ERR_NAN);
}

int mlq_fft_fwd(mlq_ctx* c, const double* u, double* fu) {
    return guard(c, [&] {
        fft64(c).fft_c2c(u, fu, -1);
        nan_scan_real_parts(fu, fft64(c).n3);
    });
}
int mlq_fft_bwd(mlq_ctx* c, const double* fu, double* u) { return guard(c, [&] { fft64(c).fft_c2c(fu, u, +1); }); }
int mlq_spectral_data(mlq_ctx* c, const double* u, int normalize, double* out) {
    return guard(c, [&] { c->solver->spectral_data_host(u, normalize, out); });
}
int mlq_state_spectral_data(mlq_ctx* c, int normalize, double* out) {
    return guard(c, [&] { c->solver->state_spectral_data(normalize, out); });
}
int mlq_summed_enstrophy(mlq_ctx* c, const double* u, double* out) {
    return guard(c, [&] { *out = c->solver->enstrophy_host(u); });
}
int mlq_dEnstrophydt(mlq_ctx* c, const double* u, double out[3]) {
    return guard(c, [&] { c->solver->dEnstrophydt_host(u, out); });
}
int mlq_pointwise_R(mlq_ctx* c, const double* u, double* out) {
    return guard(c, [&] { c->solver->pointwise_R_host(u, out); });
}
int mlq_kappa_perturbation(mlq_ctx* c, const char* type, double m1, double m2, double m3, const double* loaded,
                           unsigned long long seed, double* phi) {
    int st = 0;
    const int r = guard(c, [&] { st = fft64(c).kappa_pert(type, m1, m2, m3, loaded, seed, phi); });
    return r != MLQ_OK ? r : (st ? MLQ_ERR_IO : MLQ_OK);
}

int mlq_fft_fwdV(mlq_ctx* c, const double* u, double* fu) {
    return guard(c, [&] {
        Engine<double>& e = fft64(c);
        for (int k = 0; k < 3; ++k) {
            e.fft_c2c(u + 2 * k * e.n3, fu + 2 * k * e.n3, -1);
            nan_scan_real_parts(fu + 2 * k * e.n3, e.n3);
        }
    });
}
int mlq_fft_bwdV(mlq_ctx* c, const double* fu, double* u) {
    return guard(c, [&] {
        Engine<double>& e = fft64(c);
        for (int k = 0; k < 3; ++k) e.fft_c2c(fu + 2 * k * e.n3, u + 2 * k * e.n3, +1);
    });
}
int mlq_fft_fwdr(mlq_ctx* c, const double* u, double* fu) { return guard(c, [&] { fft64(c).fft_r2c(u, fu); }); }
int mlq_fft_bwdr(mlq_ctx* c, const double* fu, double* u) { return guard(c, [&] { fft64(c).fft_c2r(fu, u); }); }

int mlq_dealias_scalar(mlq_ctx* c, double* g, double order) {
    return guard(c, [&] { fft64(c).dealias_scalar(g, order); });
}
int mlq_gradient(mlq_ctx* c, const double* f, double* grad) {
    return guard(c, [&] { fft64(c).gradient_full(f, grad); });
}
int mlq_divergence(mlq_ctx* c, const double* u, double* div) {
    return guard(c, [&] { fft64(c).divergence_full(u, div); });
}
int mlq_laplacian(mlq_ctx* c, double* u) { return guard(c, [&] { fft64(c).laplacian_full(u); }); }
int mlq_solve_poisson(mlq_ctx* c, const double* f, double l, double* phi) {
    return guard(c, [&] { fft64(c).poisson_full(f, l, phi); });
}
int mlq_calc_uk(mlq_ctx* c, const double* u, double k, double* uk) {
    return guard(c, [&] { c->solver->calc_uk_host(u, k, uk); });
}
int mlq_divavg_free(mlq_ctx* c, double* u) { return guard(c, [&] { c->solver->divavg_host(u); }); }
int mlq_hilbert_gradient(mlq_ctx* c, double* g, double order) {
    return guard(c, [&] { c->solver->hilbert_host(g, order); });
}
int mlq_inner_product(mlq_ctx* c, const double* f, const double* g, int type, double* out) {
    return guard(c, [&] { *out = c->solver->inner_host(f, g, type); });
}
int mlq_zeroth_modes(mlq_ctx* c, const double* u, double out[3]) {
    return guard(c, [&] { c->solver->zeroth_host(u, out); });
}
int mlq_lq_norm(mlq_ctx* c, const double* u, double* norm) {
    return guard(c, [&] { *norm = c->solver->lq_norm(u); });
}
int mlq_rescale(mlq_ctx* c, double* u, double B) { return guard(c, [&] { c->solver->rescale(u, B); }); }
int mlq_normal_l2(mlq_ctx* c, const double* u, double* out) {
    return guard(c, [&] { c->solver->normal_l2(u, out); });
}
int mlq_vector_transport(mlq_ctx* c, const double* u, double q, double B, const double* eta, const double* xi,
                         double* out) {
    return guard(c, [&] { c->solver->vector_transport(u, q, B, eta, xi, out); });
}
int mlq_R_parts(mlq_ctx* c, const double* u, double out[3]) {
    return guard(c, [&] { c->solver->R_parts(u, out); });
}
int mlq_grad_l2(mlq_ctx* c, const double* u, double* v) { return guard(c, [&] { c->solver->grad_l2(u, v); }); }

int mlq_eval_J(mlq_ctx* c, const double* u, int mode, double* J) {
    return guard(c, [&] { *J = c->solver->eval_J(u, mode); });
}
int mlq_mnbrak(mlq_ctx* c, const double* phi, const double* d, double tA0, double tB0, double tau_brack[2],
               int* flag) {
    return guard(c, [&] { c->solver->mnbrak_host(phi, d, tA0, tB0, tau_brack, flag); });
}
int mlq_brent(mlq_ctx* c, const double* phi, const double* d, const double tau_brack[2], double* tau) {
    return guard(c, [&] { *tau = c->solver->brent_host(phi, d, tau_brack); });
}

int mlq_maxdlqdt(mlq_ctx* c, double* u, int start_iter, mlq_iter_cb cb, void* user, int* iterations) {
    int status = MLQ_OK;
    int st = guard(c, [&] {
        c->solver->set_start_iter(start_iter);
        c->solver->state_load(u);
        status = c->solver->state_iterate(c->p.max_iter, cb, user, iterations);
        c->solver->state_store(u);
    });
    return st != MLQ_OK ? st : status;
}

int mlq_state_load(mlq_ctx* c, const double* u) { return guard(c, [&] { c->solver->state_load(u); }); }
int mlq_state_store(mlq_ctx* c, double* u) { return guard(c, [&] { c->solver->state_store(u); }); }
int mlq_state_iterate(mlq_ctx* c, int n_iter, mlq_iter_cb cb, void* user, int* iterations) {
    int status = MLQ_OK;
    int st = guard(c, [&] { status = c->solver->state_iterate(n_iter, cb, user, iterations); });
    return st != MLQ_OK ? st : status;
}
int mlq_state_R(mlq_ctx* c, double out[3], double* lq_norm) {
    return guard(c, [&] { c->solver->state_R(out, lq_norm); });
}

int mlq_state_step(mlq_ctx* c, double* u, mlq_iter_cb cb, void* user) {
    int status = MLQ_OK;
    int st = guard(c, [&] { status = c->solver->state_step(u, cb, user); });
    return st != MLQ_OK ? st : status;
}

int mlq_profile_enable(mlq_ctx* c, int on) {
    return guard(c, [&] {
        c->solver->eng().prof_flush();
        c->solver->eng().prof_on = on != 0;
        c->solver->eng().prof_detail = on >= 2;
    });
}

int mlq_profile_report(mlq_ctx* c, char* buf, int len, int reset) {
    if (!c) return -MLQ_ERR_BADARG;
    std::string r;
    int st = guard(c, [&] { r = c->solver->eng().prof_report(reset != 0); });
    if (st != MLQ_OK) return -st;
    if (buf && len > 0) {
        std::strncpy(buf, r.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)r.size() + 1;
}

int mlq_kernel_config(mlq_ctx* c, char* buf, int len) {
    if (!c) return -MLQ_ERR_BADARG;
    std::string r;
    int st = guard(c, [&] { r = c->solver->eng().kernel_config(); });
    if (st != MLQ_OK) return -st;
    if (buf && len > 0) {
        std::strncpy(buf, r.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)r.size() + 1;
}

int mlq_seed_field(mlq_ctx* c, unsigned long long seed, double slope, double k0, double* u) {
    return guard(c, [&] { c->solver->seed_field(seed, slope, k0, u); });
}

int mlq_band_cut(int n, double order) { return band_cut_for_order(n, order); }

int mlq_seed_spectrum(int n, unsigned long long seed, double slope, double k0, double* spec, int* cut) {
    if (n < 4 || !spec) return MLQ_ERR_BADARG;
    const int c = band_cut_for_order(n, 2.0);
    Band b;
    b.n = n;
    b.cut = c;
    b.nx = c + 1;
    b.nb = 2 * c + 1;
    b.full = 0;
    seed_spectrum_host(n, seed, slope, k0, b, spec);
    if (cut) *cut = c;
    return MLQ_OK;
}

}  // extern "C"
