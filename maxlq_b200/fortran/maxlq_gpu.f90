! maxlq_gpu.f90 -- ISO_C_BINDING interface to libmaxlq_b200.so (include/maxlq.h)
!
! The module the reference's Fortran driver uses in place of fftwfunction and
! the hot-path routines of function_ops.f90 / optimization.f90.  Arrays are
! passed as assumed-size arguments: the reference's Uvec(1:n1,1:n2,1:local_N,1:3)
! with local_N = N is the layout the library takes, so no copy is needed.
! Every function returns MLQ_OK (0) or a status code (see include/maxlq.h).
! No Fortran compiler is present where this library is built, so this file is
! not compiled here; it follows the C declarations one to one.
module maxlq_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: MLQ_OK = 0, MLQ_ERR_NAN = 1, MLQ_ERR_MNBRAK_UPHILL = 2, &
       MLQ_ERR_MNBRAK_ITMAX = 3, MLQ_ERR_TAU_MAX = 4, MLQ_ERR_J_DECREASED = 5, MLQ_ERR_TIMEOUT = 6, &
       MLQ_ERR_OOM = 7, MLQ_ERR_BADARG = 8, MLQ_ERR_CUDA = 9, MLQ_ERR_NOT_BANDLIMITED = 10, MLQ_ERR_IO = 11
  integer(c_int), parameter :: MLQ_PREC_FP64 = 0, MLQ_PREC_MIXED = 1
  integer(c_int), parameter :: MLQ_J_MAXDLQDT = 0, MLQ_J_LINEMIN = 1, MLQ_J_LQNORM = 2
  integer(c_int), parameter :: MLQ_INNER_L2 = 0, MLQ_INNER_HL = 1
  integer(c_int), parameter :: MLQ_NOALLOC_MAX_N = 64

  type, bind(C) :: mlq_params
    integer(c_int) :: n
    real(c_double) :: q, B, visc, lambda1, visc_coef, press_coef
    integer(c_int) :: to_dealias, use_e_u_auto, use_e_u, dealias_e_u
    integer(c_int) :: use_tangential_gradient, use_conjugate_gradient
    integer(c_int) :: use_riemannian_geometry, normalize_gradient
    integer(c_int) :: reset_momentum_every, rolling_size, max_iter
    real(c_double) :: optim_tol
    integer(c_int) :: precision, device
  end type

  type, bind(C) :: mlq_iter_info
    integer(c_int) :: iter
    real(c_double) :: tau_a, tau, tau_b, J0, deltaJ, J1, beta, alpha
    real(c_double) :: norm_grad, norm_td0, norm_d1, u_norm_q, R, R12, R3
    real(c_double) :: ortho_check, div_check, mean_d1(3), mean_u(3)
    integer(c_int) :: n_evals, mnbrak_flag, status
    real(c_double) :: seconds
  end type

  interface
    ! ---- context (fftwfunction.f90:169-212 init_fft / fft_deallocate) ----
    subroutine mlq_default_params(p, n, q, B) bind(C)
      import; type(mlq_params) :: p; integer(c_int), value :: n; real(c_double), value :: q, B
    end subroutine
    integer(c_int) function mlq_init(ctx, p) bind(C)
      import; type(c_ptr) :: ctx; type(mlq_params), intent(in) :: p
    end function
    integer(c_int) function mlq_finalize(ctx) bind(C)
      import; type(c_ptr), value :: ctx
    end function
    type(c_ptr) function mlq_last_error(ctx) bind(C)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function mlq_set_B(ctx, B) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), value :: B
    end function
    integer(c_long_long) function mlq_kernel_launches(ctx) bind(C)
      import; type(c_ptr), value :: ctx
    end function
    integer(c_long_long) function mlq_device_bytes(ctx) bind(C)
      import; type(c_ptr), value :: ctx
    end function

    ! ---- fftwfunction.f90 ----
    integer(c_int) function mlq_fft_fwd(ctx, u, fu) bind(C)
      import; type(c_ptr), value :: ctx; complex(c_double_complex), intent(in) :: u(*)
      complex(c_double_complex) :: fu(*)
    end function
    integer(c_int) function mlq_fft_bwd(ctx, fu, u) bind(C)
      import; type(c_ptr), value :: ctx; complex(c_double_complex), intent(in) :: fu(*)
      complex(c_double_complex) :: u(*)
    end function
    integer(c_int) function mlq_fft_fwdV(ctx, u, fu) bind(C)
      import; type(c_ptr), value :: ctx; complex(c_double_complex), intent(in) :: u(*)
      complex(c_double_complex) :: fu(*)
    end function
    integer(c_int) function mlq_fft_bwdV(ctx, fu, u) bind(C)
      import; type(c_ptr), value :: ctx; complex(c_double_complex), intent(in) :: fu(*)
      complex(c_double_complex) :: u(*)
    end function
    integer(c_int) function mlq_fft_fwdr(ctx, u, fu) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*)
      complex(c_double_complex) :: fu(*)
    end function
    integer(c_int) function mlq_fft_bwdr(ctx, fu, u) bind(C)
      import; type(c_ptr), value :: ctx; complex(c_double_complex), intent(in) :: fu(*)
      real(c_double) :: u(*)
    end function

    ! ---- function_ops.f90 operators ----
    integer(c_int) function mlq_dealias_scalar(ctx, g, order) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: g(*); real(c_double), value :: order
    end function
    integer(c_int) function mlq_gradient(ctx, f, grad) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: f(*); real(c_double) :: grad(*)
    end function
    integer(c_int) function mlq_divergence(ctx, u, div) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: div(*)
    end function
    integer(c_int) function mlq_laplacian(ctx, u) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*)
    end function
    integer(c_int) function mlq_solve_poisson(ctx, f, l, phi) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: f(*); real(c_double), value :: l
      real(c_double) :: phi(*)
    end function
    integer(c_int) function mlq_calc_uk(ctx, u, k, uk) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double), value :: k
      real(c_double) :: uk(*)
    end function
    integer(c_int) function mlq_divavg_free(ctx, u) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*)
    end function
    integer(c_int) function mlq_hilbert_gradient(ctx, g, order) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: g(*); real(c_double), value :: order
    end function
    integer(c_int) function mlq_inner_product(ctx, f, g, itype, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: f(*), g(*)
      integer(c_int), value :: itype; real(c_double) :: res
    end function
    integer(c_int) function mlq_zeroth_modes(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res(3)
    end function
    integer(c_int) function mlq_lq_norm(ctx, u, norm) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: norm
    end function
    integer(c_int) function mlq_rescale(ctx, u, B) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*); real(c_double), value :: B
    end function
    integer(c_int) function mlq_normal_l2(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res(*)
    end function
    integer(c_int) function mlq_vector_transport(ctx, u, q, B, eta, xi, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*), eta(*), xi(*)
      real(c_double), value :: q, B; real(c_double) :: res(*)
    end function
    integer(c_int) function mlq_R_parts(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res(3)
    end function
    integer(c_int) function mlq_grad_l2(ctx, u, v) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: v(*)
    end function

    ! ---- diagnostics ----
    integer(c_int) function mlq_spectral_data(ctx, u, normalize, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*)
      integer(c_int), value :: normalize; real(c_double) :: res(*)
    end function
    integer(c_int) function mlq_state_spectral_data(ctx, normalize, res) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: normalize; real(c_double) :: res(*)
    end function
    integer(c_int) function mlq_summed_enstrophy(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res
    end function
    integer(c_int) function mlq_dEnstrophydt(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res(3)
    end function
    integer(c_int) function mlq_pointwise_R(ctx, u, res) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*); real(c_double) :: res(*)
    end function
    ! type: a NUL-terminated name, e.g. "create-random-poly-b"//c_null_char;
    ! loaded: c_loc of the field read from the file, or c_null_ptr
    integer(c_int) function mlq_kappa_perturbation(ctx, mytype, m1, m2, m3, loaded, seed, phi) bind(C)
      import; type(c_ptr), value :: ctx; character(kind=c_char), intent(in) :: mytype(*)
      real(c_double), value :: m1, m2, m3; type(c_ptr), value :: loaded
      integer(c_long_long), value :: seed; real(c_double) :: phi(*)
    end function

    ! ---- optimization.f90 ----
    integer(c_int) function mlq_eval_J(ctx, u, mode, J) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*)
      integer(c_int), value :: mode; real(c_double) :: J
    end function
    integer(c_int) function mlq_mnbrak(ctx, phi, d, tA0, tB0, tau_brack, flag) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: phi(*), d(*)
      real(c_double), value :: tA0, tB0; real(c_double) :: tau_brack(2); integer(c_int) :: flag
    end function
    integer(c_int) function mlq_brent(ctx, phi, d, tau_brack, tau) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: phi(*), d(*), tau_brack(2)
      real(c_double) :: tau
    end function
    integer(c_int) function mlq_maxdlqdt(ctx, u, start_iter, cb, user, iters) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*)
      integer(c_int), value :: start_iter; type(c_funptr), value :: cb; type(c_ptr), value :: user
      integer(c_int) :: iters
    end function

    ! ---- device-resident path ----
    integer(c_int) function mlq_state_load(ctx, u) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: u(*)
    end function
    integer(c_int) function mlq_state_store(ctx, u) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*)
    end function
    integer(c_int) function mlq_state_iterate(ctx, n_iter, cb, user, iters) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n_iter
      type(c_funptr), value :: cb; type(c_ptr), value :: user; integer(c_int) :: iters
    end function
    integer(c_int) function mlq_state_R(ctx, res, lq_norm) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: res(3), lq_norm
    end function
    integer(c_int) function mlq_state_step(ctx, u, cb, user) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double) :: u(*)
      type(c_funptr), value :: cb; type(c_ptr), value :: user
    end function

    ! ---- measurement ----
    integer(c_int) function mlq_profile_enable(ctx, on) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int), value :: on
    end function
    integer(c_int) function mlq_profile_report(ctx, buf, len, reset) bind(C)
      import; type(c_ptr), value :: ctx; character(kind=c_char) :: buf(*)
      integer(c_int), value :: len, reset
    end function
    integer(c_int) function mlq_kernel_config(ctx, buf, len) bind(C)
      import; type(c_ptr), value :: ctx; character(kind=c_char) :: buf(*); integer(c_int), value :: len
    end function

    ! ---- synthetic inputs ----
    integer(c_int) function mlq_seed_field(ctx, seed, slope, k0, u) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_long_long), value :: seed
      real(c_double), value :: slope, k0; real(c_double) :: u(*)
    end function
    integer(c_int) function mlq_seed_spectrum(n, seed, slope, k0, spec, cut) bind(C)
      import; integer(c_int), value :: n; integer(c_long_long), value :: seed
      real(c_double), value :: slope, k0; real(c_double) :: spec(*); integer(c_int) :: cut
    end function
    integer(c_int) function mlq_band_cut(n, order) bind(C)
      import; integer(c_int), value :: n; real(c_double), value :: order
    end function

    ! ---- gradient check (kappa_test, optimization.f90:957-1129) ----
    integer(c_int) function mlq_kappa_epsilons(n, eps) bind(C)
      import; integer(c_int), value :: n; real(c_double) :: eps(*)
    end function
    integer(c_int) function mlq_kappa_table(J0, J1, inner, n, table, adj_factor, best_index, best_kappa) bind(C)
      import; real(c_double), value :: J0, inner; real(c_double), intent(in) :: J1(*)
      integer(c_int), value :: n; real(c_double) :: table(*), adj_factor, best_kappa; integer(c_int) :: best_index
    end function

    ! ---- netCDF-3 field files (data_ops.f90) ----
    integer(c_int) function mlq_ncdf_write_field(path, n1, n2, n3, u, name1, name2, name3) bind(C)
      import; character(kind=c_char) :: path(*), name1(*), name2(*), name3(*)
      integer(c_int), value :: n1, n2, n3; real(c_double), intent(in) :: u(*)
    end function
    integer(c_int) function mlq_ncdf_read_dims(path, dims) bind(C)
      import; character(kind=c_char) :: path(*); integer(c_int) :: dims(3)
    end function
    integer(c_int) function mlq_ncdf_read_field(path, n1, n2, n3, u, name1, name2, name3) bind(C)
      import; character(kind=c_char) :: path(*), name1(*), name2(*), name3(*)
      integer(c_int), value :: n1, n2, n3; real(c_double) :: u(*)
    end function

    ! ---- no counterpart in the reference: dealias without device allocation ----
    integer(c_int) function mlq_dealias_scalar_noalloc(g, n, order) bind(C)
      import; real(c_double) :: g(*); integer(c_int), value :: n; real(c_double), value :: order
    end function
  end interface
end module maxlq_gpu
