/*
 * mlq_oracle.h -- CPU FP64 restatement of maxLq's Riemannian CG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the GPU product is
 * compared against; the product never links, loads or calls it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use it.
 *
 * Every routine restates one Fortran routine of the reference *in reference
 * order*: each dealias, derivative, Poisson solve and projection is its own
 * complex-to-complex FFT round trip followed by REAL(), exactly as
 * function_ops.f90 does, with FFTW's conventions (forward e^{-i}, unnormalised;
 * backward e^{+i} then /N^3, fftwfunction.f90:62-113).
 *
 * Parity unpinned: the reference ships no golden vectors and cannot be built
 * here (no Fortran compiler, MPI, FFTW or netCDF).  The restatement is checked
 * against analytic answers, an independent numpy transcription
 * (ref_numpy.py) and the reference's own kappa (Taylor) test instead.
 *
 * Field layout is the reference's: Fortran (n1,n2,n3[,3]) column-major, x
 * fastest, i.e. C index [c][z][y][x].  One rank holds the whole box
 * (local_N = N, local_k_offset = 0).
 */
#ifndef MLQ_ORACLE_H
#define MLQ_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int n;              /* grid points per axis (resol) */
    double q;           /* lebesgueQ */
    double B;           /* constraintB */
    double visc;        /* visc, global_variables.f90:8 */
    double lambda1;     /* lambda1, global_variables.f90:31 */
    double visc_coef;   /* viscCoefficient, global_variables.f90:113 */
    double press_coef;  /* pressureCoefficient, global_variables.f90:114 */
    int to_dealias;     /* toDealias, global_variables.f90:68 */
    int use_e_u;        /* use_e_u_instead_of_uqMinus4 (after set_e_u_or_just_u) */
    int dealias_e_u;    /* dealiase_if_mult_by_e_u, global_variables.f90:41 */
    int threads;        /* OpenMP threads (0 = runtime default) */
} orc_params;

typedef struct orc_ctx orc_ctx;

/* Per-iteration record handed back by orc_maxdlqdt (the scalars the reference
 * prints / writes in optimization.f90:420-425 and save_diagnostics_optim). */
typedef struct orc_iter_info {
    int iter;
    double tau_a, tau, tau_b;   /* tau_brack(1), tau1, tau_brack(2) */
    double J0, deltaJ, J1;
    double beta, alpha;
    double norm_grad, norm_td0, norm_d1;
    double u_norm_q;
    double R, R12, R3;          /* calc_global_dLqdt_inclParts after the update */
    int n_evals;                /* eval_J("LineMin") calls in this iteration */
    int mnbrak_flag;
} orc_iter_info;

typedef void (*orc_iter_cb)(const orc_iter_info* info, void* user);

void orc_default_params(orc_params* p, int n, double q, double B);
orc_ctx* orc_create(const orc_params* p);
void orc_destroy(orc_ctx* c);
int orc_eval_count(orc_ctx* c);  /* eval_J("LineMin") calls so far */

/* fftwfunction.f90: 3D c2c in place; dir=-1 forward (unnormalised),
 * dir=+1 backward (scaled by 1/N^3 like fftbwd).  Interleaved complex. */
void orc_fft_c2c(orc_ctx* c, double* data, int dir);

/* function_ops.f90 operators (scalar = N^3 doubles, vec = 3*N^3). */
void orc_dealias_scalar(orc_ctx* c, double* g, double order);
void orc_gradient(orc_ctx* c, const double* u, double* grad);
void orc_divergence(orc_ctx* c, const double* u, double* div);
void orc_laplacian(orc_ctx* c, double* f);
void orc_solve_poisson(orc_ctx* c, const double* f, double l, double* phi);
void orc_calc_uk(orc_ctx* c, const double* u, double k, double* uk);
void orc_unit_vector(orc_ctx* c, const double* u, double* e);
void orc_divavg_free(orc_ctx* c, double* u);
void orc_hilbert_gradient(orc_ctx* c, double* g, double order);
double orc_inner_product(orc_ctx* c, const double* f, const double* g, int htype);
double orc_field_inner(orc_ctx* c, const double* f, const double* g, int htype);
void orc_zeroth_modes(orc_ctx* c, const double* u, double out[3]);
double orc_lq_norm(orc_ctx* c, const double* u);
void orc_rescale(orc_ctx* c, double* u, double B);
void orc_normal_l2(orc_ctx* c, const double* u, double* out);
void orc_vector_transport(orc_ctx* c, const double* u, double q, double B,
                          const double* eta, const double* xi, double* out);
void orc_R_parts(orc_ctx* c, const double* u, double out[3]);
void orc_grad_l2(orc_ctx* c, const double* u, double* v);
/* mode: 0 "maxdLqdt", 1 "LineMin", 2 "||u||_q" */
double orc_eval_J(orc_ctx* c, const double* u, int mode);
int orc_mnbrak(orc_ctx* c, const double* phi, const double* d, double tA0,
               double tB0, double tau_brack[2], int* flag);
double orc_brent(orc_ctx* c, const double* phi, const double* d,
                 const double tau_brack[2]);
/* diagnostics: calculate_spectral_data (function_ops.f90:2614-2677; out is
 * 2n: kk_max then the spectrum, normalize = normalizeSpectrumByL2Norm),
 * calc_global_summed_enstrophy (2449-2467), calc_global_dEnstrophydt
 * (1417-1481; out = {R1 + R2, R1, R2}) and
 * calc_local_pointwise_dLqdt_inclParts (1224-1291; res = 3 n^3 fields
 * R1 + R2 + R3, R1 + R2, R3) */
void orc_spectral_data(orc_ctx* c, const double* u, double* out, int normalize);
double orc_summed_enstrophy(orc_ctx* c, const double* u);
void orc_dEnstrophydt(orc_ctx* c, const double* u, double out[3]);
void orc_pointwise_R(orc_ctx* c, const double* u, double* res);
/* kappa_test_pert (function_ops.f90:615-977): 1 successful, 0 a load-* type
   without its field (in = NULL), -1 unknown type */
int orc_kappa_pert(orc_ctx* c, const char* type, double m1, double m2, double m3, const double* in,
                   unsigned long long seed, double* out);
/* optimization.f90:7-514 without the file I/O and kappa tests.  u in/out.
 * Returns the number of iterations; status in *flag (0 converged/limit,
 * 1 mnbrak uphill, 2 mnbrak ITMAX, 4 tau > TAU_MAX, 5 J decreased). */
int orc_maxdlqdt(orc_ctx* c, double* u, int max_iter, double optim_tol,
                 int start_iter, orc_iter_cb cb, void* user, int* flag);

#ifdef __cplusplus
}
#endif
#endif
