// solver.cuh -- maxdLqdt / mnbrak / brent on the device-resident state.
//
// Scalar control (bracketing, Brent, Polak-Ribiere beta, stop test) runs on
// the host in FP64 exactly as optimization.f90 does; every function value,
// gradient, inner product and update runs on the GPU against the FP64 state
// spectra.  A line-search trial J(tau) = -R(B (u+tau d)/||u+tau d||_q) is one
// R evaluation at u + tau d and the homogeneity
// R(c w) = c^q (R1+R2)(w) + c^(q+1) R3(w) (every term of R is a product of
// q or q+1 powers of the field), which is also how J1 after the update is
// obtained from the accepted trial.
#pragma once

#include <chrono>
#include <map>

#include "engine.cuh"

namespace mlq {

struct Trial {
    double lqq;   // ||w||_q^q
    double R[3];  // R, R1+R2, R3 at w (unscaled)
};

class SolverBase {
   public:
    virtual ~SolverBase() {}
    virtual EngineBase& eng() = 0;
    // host-array entry points (each loads its input as a band-limited state)
    virtual void R_parts(const double* u, double out[3]) = 0;
    virtual double eval_J(const double* u, int mode) = 0;
    virtual void grad_l2(const double* u, double* v) = 0;
    virtual double lq_norm(const double* u) = 0;
    virtual void rescale(double* u, double B) = 0;
    virtual void normal_l2(const double* u, double* out) = 0;
    virtual void vector_transport(const double* u, double q, double B, const double* eta, const double* xi,
                                  double* out) = 0;
    virtual void hilbert_host(double* g, double order) = 0;
    virtual void divavg_host(double* g) = 0;
    virtual double inner_host(const double* f, const double* g, int type) = 0;
    virtual void zeroth_host(const double* u, double out[3]) = 0;
    virtual void calc_uk_host(const double* u, double k, double* out) = 0;
    // diagnostics of a host field, and the spectrum of the resident state
    virtual void spectral_data_host(const double* u, int normalize, double* out) = 0;
    virtual void state_spectral_data(int normalize, double* out) = 0;
    virtual double enstrophy_host(const double* u) = 0;
    virtual void dEnstrophydt_host(const double* u, double out[3]) = 0;
    virtual void pointwise_R_host(const double* u, double* out) = 0;
    virtual int mnbrak_host(const double* phi, const double* d, double tA0, double tB0, double br[2], int* flag) = 0;
    virtual double brent_host(const double* phi, const double* d, const double br[2]) = 0;
    // resident state
    virtual void state_load(const double* u) = 0;
    virtual void state_store(double* u) = 0;
    virtual int state_iterate(int n_iter, mlq_iter_cb cb, void* user, int* iters) = 0;
    virtual void state_R(double out[3], double* lqn) = 0;
    virtual int state_step(double* u, mlq_iter_cb cb, void* user) = 0;
    virtual void seed_field(unsigned long long seed, double slope, double k0, double* u) = 0;
    virtual void set_B(double B) = 0;
    virtual void set_start_iter(int s) = 0;
    int eval_count = 0;
};

std::unique_ptr<SolverBase> make_solver(const mlq_params& p);
std::unique_ptr<EngineBase> make_fft_engine(const mlq_params& p);

}  // namespace mlq
