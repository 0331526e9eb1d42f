! dqmc_gpu_f.f90 -- iso_c_binding interface to libdqmc_gpu.so for the
! Fortran reference (sun-hubbard, YuanyueChen/sunhubbardmy).
!
! A maintainer adds this module to the reference's src/ and calls it under
! #ifdef GPU from dqmc_ft_ctrl.f90 / dqmc_ft_core (finite temperature) and
! dqmc_proj_ctrl.f90 / dqmc_proj_core (projective).  Each interface mirrors one
! declaration of include/dqmc_gpu.h (same name, argument order and types);
! the derived types mirror dqmc_params and dqmc_diag field by field, so a
! call never writes past a Fortran variable.  Integer arguments passed by
! value are C int; arrays are passed by reference in the reference's own
! column-major layouts (conf(nsites, ltrot), gf%blk1(ndim, ndim), ...).
! Every function returns 0 or a negative DQMC_E* code; the constants below
! repeat the header's.
module dqmc_gpu_f
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: DQMC_OK = 0, DQMC_EINVAL = -1, DQMC_ECUDA = -2, DQMC_ENOMEM = -3
  integer(c_int), parameter :: DQMC_ESTATE = -4, DQMC_ENUMERIC = -5, DQMC_EWRAP = -6
  integer(c_int), parameter :: DQMC_LATT_SQUARE = 1, DQMC_LATT_HONEYCOMB = 2, DQMC_LATT_CHAIN = 3, &
                                DQMC_LATT_CUBIC = 4, DQMC_LATT_R_CUBIC = 5
  integer(c_int), parameter :: DQMC_UPD_FAST = 0, DQMC_UPD_DELAY = 1, DQMC_UPD_SUBMATRIX = 2
  integer(c_int), parameter :: DQMC_KIN_CHECKERBOARD = 0, DQMC_KIN_FFT = 1, DQMC_KIN_DENSE = 2
  integer(c_int), parameter :: DQMC_HS_EXACT = 0, DQMC_HS_GENERAL4 = 1

  ! mirror of dqmc_params in include/dqmc_gpu.h (same field order)
  type, bind(C) :: dqmc_params_c
     integer(c_int32_t) :: lattice, l1, l2
     real(c_double)     :: beta, dtau, rt, t2, t3, nu, mu, rhub, rv, alpha, theta
     real(c_double)     :: xmag, flux_x, flux_y, dimer, rndness
     integer(c_int32_t) :: nflr, lproju, lstabilize
     integer(c_int32_t) :: nwrap, nsweep, nbin, nublock
     integer(c_int32_t) :: update, kinetic, hs
     integer(c_int32_t) :: proj, lprojv, obs_mid_len
     integer(c_int32_t) :: ndim, lq, ltrot, nst, ne, lcomp
     integer(c_int32_t) :: ltau, ntdm
     real(c_double)     :: dyntau
     integer(c_int32_t) :: l3
     real(c_double)     :: rtd
     real(c_double)     :: rhub_plq
     integer(c_int32_t) :: lprojplqu
  end type

  ! mirror of dqmc_diag (same field order)
  type, bind(C) :: dqmc_diag_c
     real(c_double) :: phase_re, phase_im, logweight_re, logweight_im
     real(c_double) :: max_wrap_error, max_phasediff, avglog10error_sum, logcount
     real(c_double) :: avgexpphasediff_sum, accepted, proposed, nobs
     real(c_double) :: accepted_v, proposed_v
     real(c_double) :: blk_proposed, blk_stage1, blk_accepted, blk_sum_logratio
     real(c_double) :: blk_err_learned, blk_err_zero
     real(c_double) :: max_dyn_error, dyn_log10_sum, dyn_count
     real(c_double) :: info, restabilized
     real(c_double) :: near_ties
     real(c_double) :: accepted_plq, proposed_plq
  end type

  interface
     ! make_tables (src/model_para.f90:334-453)
     integer(c_int) function dqmc_params_derive(p) bind(C)
       import; type(dqmc_params_c) :: p
     end function
     ! dqmc_start: set_h0conf, set_conf, input_conf, allocate_core (src/dqmc_ft_ctrl.f90:9-45)
     integer(c_int) function dqmc_gpu_create(p, np, nch, seeds, draw, h) bind(C)
       import; type(dqmc_params_c) :: p(*); integer(c_int), value :: np, nch
       integer(c_int32_t) :: seeds(*); integer(c_int), value :: draw; type(c_ptr) :: h
     end function
     integer(c_int) function dqmc_gpu_destroy(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     type(c_ptr) function dqmc_gpu_last_error() bind(C)
       import
     end function
     ! uconf%conf (input_conf / output_conf)
     integer(c_int) function dqmc_gpu_set_conf(h, c, conf) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: conf(*)
     end function
     integer(c_int) function dqmc_gpu_get_conf(h, c, conf) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: conf(*)
     end function
     ! gf%blk1
     integer(c_int) function dqmc_gpu_get_green(h, c, g) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: g(*)
     end function
     integer(c_int) function dqmc_gpu_set_green(h, c, g) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: g(*)
     end function
     ! Ust(n), Dst(n), Vst(n), logdetQst(n) (src/dqmc_ft_core.f90:11-19)
     integer(c_int) function dqmc_gpu_get_stack(h, c, n, u, d, v, logdetq) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c, n
       complex(c_double_complex) :: u(*); real(c_double) :: d(*); complex(c_double_complex) :: v(*)
       complex(c_double_complex) :: logdetq
     end function
     integer(c_int) function dqmc_gpu_set_stack(h, c, n, u, d, v, logdetq) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c, n
       complex(c_double_complex) :: u(*); real(c_double) :: d(*); complex(c_double_complex) :: v(*)
       complex(c_double_complex) :: logdetq
     end function
     ! numerical checks: the reference's stop on a failed inversion becomes DQMC_ENUMERIC
     integer(c_int) function dqmc_gpu_set_checks(h, wrap_tol, restabilize) bind(C)
       import; type(c_ptr), value :: h; real(c_double), value :: wrap_tol; integer(c_int), value :: restabilize
     end function
     ! dqmc_ft_sweep_start_0b, dqmc_ft_sweep_b0 / _0b
     integer(c_int) function dqmc_gpu_sweep_start(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     integer(c_int) function dqmc_gpu_sweep_b0(h, lupd, lmeas) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: lupd, lmeas
     end function
     integer(c_int) function dqmc_gpu_sweep_0b(h, lupd, lmeas) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: lupd, lmeas
     end function
     integer(c_int) function dqmc_gpu_sweeps(h, n, lmeas) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: n, lmeas
     end function
     ! obser_init, equaltime_measure bins, diagnostics
     integer(c_int) function dqmc_gpu_obser_init(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     integer(c_int) function dqmc_gpu_nbins(h, c) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c
     end function
     integer(c_int) function dqmc_gpu_get_bins(h, c, out) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: out(*)
     end function
     integer(c_int) function dqmc_gpu_get_diag(h, c, d) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; type(dqmc_diag_c) :: d
     end function
     integer(c_int) function dqmc_gpu_reset_diag(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     ! SFMT state of one chain (spring_sfmt_*, lib/m_spring.f90:187-379)
     integer(c_int) function dqmc_gpu_get_rng(h, c, state) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: state(*)
     end function
     integer(c_int) function dqmc_gpu_set_rng(h, c, state) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: state(*)
     end function
     ! type-bound operators of h0conf / uconf on the current G
     integer(c_int) function dqmc_gpu_h0_prop(h, op, nf) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: op, nf
     end function
     integer(c_int) function dqmc_gpu_u_prop(h, op, nt) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: op, nt
     end function
     integer(c_int) function dqmc_gpu_update(h, nt) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: nt
     end function
     integer(c_int) function dqmc_gpu_measure(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     integer(c_int) function dqmc_gpu_set_phase(h, c, re, im) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; real(c_double), value :: re, im
     end function
     ! -DTIMING breakdown (dqmc_timing / dqmc_end)
     integer(c_int) function dqmc_gpu_sweep_profile(h, nsweeps, lmeas, ms, groups) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: nsweeps, lmeas
       real(c_double) :: ms(*); integer(c_int) :: groups(*)
     end function
     ! unequal-time measurement (ltau)
     integer(c_int) function dqmc_gpu_sweep_dyn(h) bind(C)
       import; type(c_ptr), value :: h
     end function
     integer(c_int) function dqmc_gpu_get_dyn_bins(h, c, out) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: out(*)
     end function
     ! projective path (params%proj = 1)
     integer(c_int) function dqmc_gpu_set_vconf(h, c, v) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: v(*)
     end function
     integer(c_int) function dqmc_gpu_get_vconf(h, c, v) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: v(*)
     end function
     integer(c_int) function dqmc_gpu_set_conf_plq(h, c, v) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: v(*)
     end function
     integer(c_int) function dqmc_gpu_get_conf_plq(h, c, v) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; integer(c_int32_t) :: v(*)
     end function
     integer(c_int) function dqmc_gpu_get_trial(h, c, proj, w) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: proj(*)
       real(c_double) :: w(*)
     end function
     integer(c_int) function dqmc_gpu_set_trial(h, c, proj) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c; complex(c_double_complex) :: proj(*)
     end function
     integer(c_int) function dqmc_gpu_get_proj(h, c, ur, ul, ulrinv) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c
       complex(c_double_complex) :: ur(*), ul(*), ulrinv(*)
     end function
     integer(c_int) function dqmc_gpu_set_proj(h, c, ur, ul, ulrinv) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: c
       complex(c_double_complex) :: ur(*), ul(*), ulrinv(*)
     end function
     integer(c_int) function dqmc_gpu_proj_update(h, nt, nf) bind(C)
       import; type(c_ptr), value :: h; integer(c_int), value :: nt, nf
     end function
     integer(c_int) function dqmc_gpu_proj_green(h) bind(C)
       import; type(c_ptr), value :: h
     end function
  end interface
end module dqmc_gpu_f
