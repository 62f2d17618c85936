/*
 * maxlq.h -- C ABI of the B200 engine for maxLq's Riemannian CG search.
 *
 * Drop-in boundary for the reference's hot path (uniFabiB/maxLq): the Fortran
 * driver keeps calling the same subroutine surface; an ISO_C_BINDING module
 * (maxlq_b200/fortran/maxlq_gpu.f90) binds each routine below.
 *
 * Conventions (identical to the reference):
 *   - unit box [0,1]^3, K_j = 2*pi*j (initialize.f90:170-192), dV = 1/N^3;
 *   - a vector field is a host array of 3*N^3 doubles laid out as the Fortran
 *     array U(1:n1,1:n2,1:n3,1:3): column-major, x fastest, component slowest;
 *     a scalar field is N^3 doubles (n1,n2,n3);
 *   - complex arrays are interleaved (re,im) pairs, Fortran complex(8);
 *   - forward FFTs are unnormalised (FFTW_FORWARD), backward ones are scaled
 *     by 1/N^3 (fftwfunction.f90:109, 160).
 * Every call returns an int status (MLQ_OK = 0) instead of the reference's
 * `stop 1`; mlq_last_error() gives the message.  Calls on one context are not
 * thread-safe; each context owns one CUDA stream on one device.
 */
#ifndef MAXLQ_H
#define MAXLQ_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MLQ_OK 0
#define MLQ_ERR_NAN 1             /* NaN found (fftwfunction.f90:78-89, function_ops.f90:1843-1854) */
#define MLQ_ERR_MNBRAK_UPHILL 2   /* mnbrak myflag=1 (optimization.f90:685-688) */
#define MLQ_ERR_MNBRAK_ITMAX 3    /* mnbrak myflag=2 (optimization.f90:769-773) */
#define MLQ_ERR_TAU_MAX 4         /* tau > TAU_MAX (optimization.f90:310-314) */
#define MLQ_ERR_J_DECREASED 5     /* cost functional not increasing (optimization.f90:351-366) */
#define MLQ_ERR_TIMEOUT 6         /* a bounded device wait gave up */
#define MLQ_ERR_OOM 7             /* device allocation failed */
#define MLQ_ERR_BADARG 8          /* invalid argument / unsupported configuration */
#define MLQ_ERR_CUDA 9            /* other CUDA runtime error */
#define MLQ_ERR_NOT_BANDLIMITED 10 /* input field has modes outside the 2/3 dealiasing cube */
#define MLQ_ERR_IO 11             /* a file could not be opened, read or written, or is not netCDF-3 */

/* precision of the transform pipeline; CG state and reductions are FP64 */
#define MLQ_PREC_FP64 0
#define MLQ_PREC_MIXED 1 /* FP32 fields and FFTs, FP64 reductions and control */

/* eval_J modes (optimization.f90:533-545) */
#define MLQ_J_MAXDLQDT 0 /* "maxdLqdt": R(u) */
#define MLQ_J_LINEMIN 1  /* "LineMin": -R(B u/||u||_q) */
#define MLQ_J_LQNORM 2   /* "||u||_q" */

/* inner products (function_ops.f90:3404-3503) */
#define MLQ_INNER_L2 0
#define MLQ_INNER_HL 1 /* "H_l^(3/2-1/q)" */

typedef struct mlq_ctx mlq_ctx;

/* Mirrors the module globals the hot path reads (global_variables.f90:8-86,
 * initialize.f90:88-127).  Fill with mlq_default_params() first. */
typedef struct mlq_params {
    int n;                     /* resol: grid points per axis */
    double q;                  /* lebesgueQ */
    double B;                  /* constraintB */
    double visc;               /* visc (8) */
    double lambda1;            /* lambda1 (31) */
    double visc_coef;          /* viscCoefficient (113) */
    double press_coef;         /* pressureCoefficient (114) */
    int to_dealias;            /* toDealias (68); only 1 is supported */
    int use_e_u_auto;          /* use_e_u_auto_for_q_less_4 (39) */
    int use_e_u;               /* use_e_u_instead_of_uqMinus4 (40) when auto is off */
    int dealias_e_u;           /* dealiase_if_mult_by_e_u (41); only 1 is supported */
    int use_tangential_gradient; /* (32) */
    int use_conjugate_gradient;  /* (33) */
    int use_riemannian_geometry; /* (34) */
    int normalize_gradient;      /* (38) */
    int reset_momentum_every;    /* resetMomentumTermEveryXiterations (35) */
    int rolling_size;            /* toleranceRollingAverageSize (36) */
    int max_iter;                /* MAX_ITER (26) */
    double optim_tol;            /* OPTIM_TOL (initialize.f90:96-100) */
    int precision;               /* MLQ_PREC_FP64 or MLQ_PREC_MIXED */
    int device;                  /* CUDA device ordinal */
} mlq_params;

/* Scalars of one CG iteration, everything the reference prints or writes
 * (optimization.f90:420-425, save_diagnostics_optim, the optim_msg codes). */
typedef struct mlq_iter_info {
    int iter;
    double tau_a, tau, tau_b;      /* tau_brack(1), tau1, tau_brack(2) */
    double J0, deltaJ, J1;
    double beta, alpha;
    double norm_grad, norm_td0, norm_d1; /* H-norms printed at 245-247 */
    double u_norm_q;               /* ||u||_q after the update (421) */
    double R, R12, R3;             /* calc_global_dLqdt_inclParts (423) */
    double ortho_check;            /* test1 at 180 (msg 42 when > 1e-12) */
    double div_check;              /* test1 at 189 (msg 43 when > 1e-15) */
    double mean_d1[3], mean_u[3];  /* calc0thFourierModes (251-261, msg 44) */
    int n_evals;                   /* eval_J("LineMin") calls this iteration */
    int mnbrak_flag;
    int status;                    /* MLQ_OK or the code that ends the loop */
    double seconds;                /* device wall time of this iteration */
} mlq_iter_info;

typedef void (*mlq_iter_cb)(const mlq_iter_info* info, void* user);

/* ---- context (fftwfunction.f90:169-212 init_fft / fft_deallocate) ------- */
void mlq_default_params(mlq_params* p, int n, double q, double B);
int mlq_init(mlq_ctx** ctx, const mlq_params* p);
int mlq_finalize(mlq_ctx* ctx);
const char* mlq_last_error(const mlq_ctx* ctx);
int mlq_set_B(mlq_ctx* ctx, double B); /* constraintB between continuation steps */
/* number of engine kernel launches so far (for launch accounting) */
long long mlq_kernel_launches(const mlq_ctx* ctx);
/* device bytes held by the context */
long long mlq_device_bytes(const mlq_ctx* ctx);

/* ---- fftwfunction.f90 ---------------------------------------------------- */
/* fftfwd / fftbwd (62-113): 3D c2c of N^3 complex(8), normal order.
 * mlq_fft_fwd returns MLQ_ERR_NAN when the real part of an output is NaN
 * (fftfwd's scan, 78-89). */
int mlq_fft_fwd(mlq_ctx* ctx, const double* u, double* fu);
int mlq_fft_bwd(mlq_ctx* ctx, const double* fu, double* u);
/* fftfwdV / fftbwdV (24-58): the three components of a complex(8)
 * (N,N,N,3) field, each through fftfwd / fftbwd */
int mlq_fft_fwdV(mlq_ctx* ctx, const double* u, double* fu);
int mlq_fft_bwdV(mlq_ctx* ctx, const double* fu, double* u);
/* fftfwdr / fftbwdr (118-164): real (N,N,N) <-> complex (N/2+1,N,N) */
int mlq_fft_fwdr(mlq_ctx* ctx, const double* u, double* fu);
int mlq_fft_bwdr(mlq_ctx* ctx, const double* fu, double* u);

/* ---- function_ops.f90 operators ------------------------------------------ */
/* order non-finite or below -1 (no mode kept) -> MLQ_ERR_BADARG */
int mlq_dealias_scalar(mlq_ctx* ctx, double* g, double order);            /* 3332-3350 */
int mlq_gradient(mlq_ctx* ctx, const double* f, double* grad);             /* 3147-3195 */
int mlq_divergence(mlq_ctx* ctx, const double* u, double* div);            /* 3200-3243 */
int mlq_laplacian(mlq_ctx* ctx, double* u);                                /* 3248-3282 */
int mlq_solve_poisson(mlq_ctx* ctx, const double* f, double l, double* phi); /* 1951-1996 */
int mlq_calc_uk(mlq_ctx* ctx, const double* u, double k, double* uk);      /* 2324-2343 */
int mlq_divavg_free(mlq_ctx* ctx, double* u);                              /* 2843-2918 */
int mlq_hilbert_gradient(mlq_ctx* ctx, double* g, double order);           /* 3583-3627 */
int mlq_inner_product(mlq_ctx* ctx, const double* f, const double* g, int type, double* out); /* 3557-3577 */
int mlq_zeroth_modes(mlq_ctx* ctx, const double* u, double out[3]);        /* 3048-3094 */
int mlq_lq_norm(mlq_ctx* ctx, const double* u, double* norm);              /* 1675-1692 */
int mlq_rescale(mlq_ctx* ctx, double* u, double B);                        /* 1699-1709 */
int mlq_normal_l2(mlq_ctx* ctx, const double* u, double* out);             /* 984-1006 */
int mlq_vector_transport(mlq_ctx* ctx, const double* u, double q, double B,
                         const double* eta, const double* xi, double* out); /* 1716-1768 */
int mlq_R_parts(mlq_ctx* ctx, const double* u, double out[3]);             /* 1392-1405 */
int mlq_grad_l2(mlq_ctx* ctx, const double* u, double* v);                 /* GradL2ForLq 1066-1211 */

/* ---- diagnostics (maxdLpdt.f90:263-299, optimization.f90:119-123, 377-384) -- */
/* calculate_spectral_data (function_ops.f90:2614-2677): out is the Fortran
 * array spectral_data(1:n, 1:2), out[0..n) = kk_max = 2 pi i (i = 1..n) and
 * out[n..2n) the energy of fftfwd(u) in the shell kk_max - 2 pi < |K| <=
 * kk_max; normalize = normalizeSpectrumByL2Norm (global_variables.f90:76)
 * scales it by <u,u>_L2 / (2 pi sum).  u must be band-limited like every field
 * of the path (MLQ_ERR_NOT_BANDLIMITED otherwise). */
int mlq_spectral_data(mlq_ctx* ctx, const double* u, int normalize, double* out);
/* the same for the resident state (calculateSaveSpectrum(uvec) inside the loop) */
int mlq_state_spectral_data(mlq_ctx* ctx, int normalize, double* out);
/* calc_global_summed_enstrophy (2449-2467): 1/2 ||curl u||_2^2 */
int mlq_summed_enstrophy(mlq_ctx* ctx, const double* u, double* out);
/* calc_global_dEnstrophydt (1417-1481): out = {R1 + R2, R1, R2} with
 * R1 = -viscCoefficient visc ||Lap u||^2, R2 = <P2((u.grad) u), Lap u> */
int mlq_dEnstrophydt(mlq_ctx* ctx, const double* u, double out[3]);
/* calc_local_pointwise_dLqdt_inclParts (1224-1291): out is the (n,n,n,3)
 * field (R1 + R2 + R3, R1 + R2, R3) saved as "Ru" (maxdLpdt.f90:299) */
int mlq_pointwise_R(mlq_ctx* ctx, const double* u, double* out);
/* kappa_test_pert (function_ops.f90:615-977): the gradient check's
 * perturbation phi_pert (n,n,n,3) of the reference's type name ("sine",
 * "divfree-sine", "load-te0080", "load-random-a|b", "load-random-smooth-a|b",
 * "load-k-random-a|b", "load-random-poly-a|b", "load-random-exp-a|b",
 * "create-random-poly-b", "save-random"), full band, FP64 on the device.
 * loaded: the field a load-* type reads from its netCDF file
 * (mlq_ncdf_read_field), NULL when the file is missing: the field is then
 * formed from zeros and MLQ_ERR_IO returned (the reference's
 * successful = .false.).  The random fields come from a seeded generator
 * (splitmix64 of seed and the element index) where the reference calls an
 * unseeded random_number.  Unknown type: MLQ_ERR_BADARG. */
int mlq_kappa_perturbation(mlq_ctx* ctx, const char* type, double m1, double m2, double m3, const double* loaded,
                           unsigned long long seed, double* phi);

/* ---- optimization.f90 ---------------------------------------------------- */
int mlq_eval_J(mlq_ctx* ctx, const double* u, int mode, double* J);        /* 520-547 */
int mlq_mnbrak(mlq_ctx* ctx, const double* phi, const double* d, double tA0, double tB0,
               double tau_brack[2], int* flag);                            /* 613-778 */
int mlq_brent(mlq_ctx* ctx, const double* phi, const double* d, const double tau_brack[2],
              double* tau);                                                /* 784-951 */
/* maxdLqdt (7-514): the whole CG loop for the current B; u in/out.
 * start_iter = optimizationIterOffset for a resumed run (81-85). */
int mlq_maxdlqdt(mlq_ctx* ctx, double* u, int start_iter, mlq_iter_cb cb, void* user, int* iterations);

/* ---- device-resident path (no PCIe inside the loop) ---------------------- */
/* Load u (host, reference layout) into the context's resident state. */
int mlq_state_load(mlq_ctx* ctx, const double* u);
int mlq_state_store(mlq_ctx* ctx, double* u);
/* Run up to n_iter CG iterations on the resident state (CG memory kept across
 * calls); the first call after mlq_state_load performs the pre-loop steps
 * (optimization.f90:61-78). */
int mlq_state_iterate(mlq_ctx* ctx, int n_iter, mlq_iter_cb cb, void* user, int* iterations);
/* Resident-state R(u) parts and ||u||_q. */
int mlq_state_R(mlq_ctx* ctx, double out[3], double* lq_norm);
/* One CG iteration on u in host memory: u (reference layout) replaces the
 * resident field, the CG memory of earlier steps is kept, one iteration runs
 * and the updated u is copied back.  The first step performs the pre-loop
 * steps like mlq_state_iterate. */
int mlq_state_step(mlq_ctx* ctx, double* u, mlq_iter_cb cb, void* user);

/* ---- measurement ----------------------------------------------------------- */
/* Per-kernel CUDA-event timing on the context's stream (off by default).
 * on = 2 also keys each x-stage launch by its fused pointwise functor. */
int mlq_profile_enable(mlq_ctx* ctx, int on);
/* JSON object {kernel: [launches, total_ms, algorithmic_bytes]} of the launches
 * since the last reset; resets when reset != 0.  Returns the length needed. */
int mlq_profile_report(mlq_ctx* ctx, char* buf, int len, int reset);
/* JSON object describing the pass kernels the context runs: precision,
 * kernel family (compile-time / register / shared-memory Stockham) and the
 * y/z tile shapes the autotuner chose with their timings.  No counterpart in
 * the reference (it has a single FFTW path).  Returns the length needed. */
int mlq_kernel_config(mlq_ctx* ctx, char* buf, int len);

/* ---- synthetic inputs ------------------------------------------------------ */
/* Seeded divergence-free, 2/3-dealiased field with amplitude
 * |j|^-slope * exp(-(|j|/k0)^2) (Philox-4x32-10, key = seed, counter =
 * (jx, jy, jz, component)); written to u in the reference layout.  Not
 * rescaled: maxdLqdt rescales to ||u||_q = B itself (optimization.f90:61). */
int mlq_seed_field(mlq_ctx* ctx, unsigned long long seed, double slope, double k0, double* u);
/* Host-only: the same field as a pruned half spectrum, for checkers.  Layout
 * [3][2c+1 kz][2c+1 ky][c+1 kx] complex, c = 2/3 cut of n, compact index order
 * 0..c, -c..-1.  Returns c via *cut. */
int mlq_seed_spectrum(int n, unsigned long long seed, double slope, double k0, double* spec, int* cut);
int mlq_band_cut(int n, double order); /* largest |j| kept by a dealias of that order */

/* ---- gradient check (host only) -------------------------------------------- */
/* kappa_test (optimization.f90:957-1129): eps[i-1] = 10^(-7 - n/2 + i),
 * i = 1..n (the reference uses n = 16, 1037-1038) */
int mlq_kappa_epsilons(int n, double* eps);
/* the kappa table from J0 = J(phi), J1[i-1] = J(phi + eps_i phi_pert) and
 * inner = <grad J, phi_pert> (1027-1081): table is n x 5, row-major, rows
 * (eps, inner, J1 - J0, kappa, adjusted kappa) as kappaArray; *adj_factor is
 * the divisor of the adjusted column, *best_index (1-based) and *best_kappa
 * the reference's best kappa.  n >= 5. */
int mlq_kappa_table(double J0, const double* J1, double inner, int n, double* table, double* adj_factor,
                    int* best_index, double* best_kappa);

/* ---- netCDF-3 classic field files (host only, no libnetcdf) ---------------- */
/* save_field_R3toR3_ncdf (data_ops.f90:362-487, the parallel_data layout the
 * reference uses for N >= 16): a CDF-1 file with dimensions "x" = n1, "y" = n2
 * and an unlimited "z" holding n3 records, and three NC_DOUBLE record
 * variables name1..3 of dimensions (z, y, x), no attributes.  u is the
 * (n1, n2, n3, 3) column-major host field. */
int mlq_ncdf_write_field(const char* path, int n1, int n2, int n3, const double* u, const char* name1,
                         const char* name2, const char* name3);
/* the lengths of the dimensions "x", "y", "z" of a classic or 64-bit-offset
 * netCDF file (data_ops.f90:1237-1265) */
int mlq_ncdf_read_dims(const char* path, int dims[3]);
/* read_field_R3toR3_ncdf (data_ops.f90:1198-1397): the NC_DOUBLE variables
 * name1..3 of dimensions (z, y, x), z a record or a fixed dimension, into the
 * (n1, n2, n3, 3) column-major host field u.  MLQ_ERR_BADARG when a variable
 * is missing, not NC_DOUBLE or of other dimensions. */
int mlq_ncdf_read_field(const char* path, int n1, int n2, int n3, double* u, const char* name1, const char* name2,
                        const char* name3);

/* ---- allocation-free variant ----------------------------------------------- */
/* No counterpart in the reference.  dealias_scalar for callers that cannot
 * allocate device memory -- a host program whose device memory is owned by
 * another runtime, or code that must not trigger an allocation (which can
 * synchronise the device) -- so it needs no context: g is the host scalar
 * field (n,n,n), dealiased in place exactly as mlq_dealias_scalar does.  All
 * device memory it uses is one static array of about 6.4 MiB that every GPU
 * loading this library holds until exit, which limits n to
 * MLQ_NOALLOC_MAX_N; larger n, a non-finite order and an order below -1 are
 * rejected with MLQ_ERR_BADARG (message on stderr).  The call works in the
 * calling thread's current device and context and looks up the array's
 * address there on every call.  It copies with synchronous cudaMemcpy on the
 * legacy default stream, so it must not be called during stream capture.
 * Calls share the array: calls that overlap on the GPU (from several host
 * threads) race.  Every call overwrites all of the array it reads, so
 * nothing carries over from the previous call. */
#define MLQ_NOALLOC_MAX_N 64
int mlq_dealias_scalar_noalloc(double* g, int n, double order);

#ifdef __cplusplus
}
#endif
#endif /* MAXLQ_H */
