! lmm_stokes_iface.f90 - iso_c_binding interface to liblmmstokes
! (include/lmm_stokes.h).  The derived types mirror the C structs field by
! field; the interfaces bind the C-ABI entry points.  Shipped as source: it
! is compiled into the application together with gmres_lmm.f90, which
! replaces src_gmres/gmres.f90.
module lmm_stokes_iface

  use iso_c_binding

  implicit none

  integer(c_int), parameter :: LMM_OK = 0
  integer(c_int), parameter :: LMM_LAYOUT_COMPACT = 0
  integer(c_int), parameter :: LMM_LAYOUT_BOXLIB = 1
  integer(c_int), parameter :: LMM_METHOD_GMRES = 0
  integer(c_int), parameter :: LMM_METHOD_FGMRES = 1
  integer(c_int), parameter :: LMM_PRECISION_FP64 = 0
  integer(c_int), parameter :: LMM_PRECISION_FP32 = 1
  integer(c_int), parameter :: LMM_BC_PERIODIC = -1
  integer(c_int), parameter :: LMM_BC_NO_SLIP_WALL = 100, LMM_BC_SLIP_WALL = 200
  integer(c_int), parameter :: LMM_HISTORY_MAX = 512

  type, bind(c) :: lmm_grid
     integer(c_int) :: dm
     integer(c_int) :: n(3)
     real(c_double) :: dx
     integer(c_int) :: bc_lo(3)
     integer(c_int) :: bc_hi(3)
  end type lmm_grid

  ! one field per variable of probin_gmres_module (probin_gmres.f90:13-22),
  ! then visc_type and the additions of the library, in the C order
  type, bind(c) :: lmm_knobs
     integer(c_int) :: precon_type, visc_schur_approx
     real(c_double) :: p_norm_weight, scale_factor
     integer(c_int) :: mg_verbose, cg_verbose, mg_max_vcycles, mg_minwidth, mg_bottom_solver
     integer(c_int) :: mg_nsmooths_down, mg_nsmooths_up, mg_nsmooths_bottom, mg_max_bottom_nlevels
     real(c_double) :: mg_rel_tol
     integer(c_int) :: stag_mg_verbosity, stag_mg_max_vcycles, stag_mg_minwidth, stag_mg_bottom_solver
     integer(c_int) :: stag_mg_nsmooths_down, stag_mg_nsmooths_up, stag_mg_nsmooths_bottom
     integer(c_int) :: stag_mg_max_bottom_nlevels
     real(c_double) :: stag_mg_omega
     integer(c_int) :: stag_mg_smoother
     real(c_double) :: stag_mg_rel_tol
     real(c_double) :: gmres_rel_tol, gmres_abs_tol
     integer(c_int) :: gmres_verbose, gmres_max_outer, gmres_max_inner, gmres_max_iter, gmres_min_iter
     integer(c_int) :: visc_type
     integer(c_int) :: method, precision, learned_stage
     integer(c_int) :: tail_cells, tail_smem_kb, use_graphs, smoother_fusion, l2_persist
     integer(c_int) :: orthogonalization, host_wait
     integer(c_int) :: ensemble_batch
     integer(c_int) :: smoother_tma, smoother_tma_slabs, smoother_tma_cells, smoother_order
     integer(c_int) :: autotune, residual_fusion, uniform_alpha
     integer(c_int) :: smoother_fusion_cells
  end type lmm_knobs

  type, bind(c) :: lmm_fields_in
     type(c_ptr) :: b_u(3)
     type(c_ptr) :: b_p
     type(c_ptr) :: alpha_fc(3)
     type(c_ptr) :: beta
     type(c_ptr) :: beta_ed(3)
     type(c_ptr) :: gamma
     integer(c_int) :: layout
     integer(c_int) :: ng_b_u, ng_b_p, ng_alpha, ng_beta, ng_beta_ed, ng_gamma
  end type lmm_fields_in

  type, bind(c) :: lmm_fields_out
     type(c_ptr) :: x_u(3)
     type(c_ptr) :: x_p
     integer(c_int) :: layout
     integer(c_int) :: ng_x_u, ng_x_p
  end type lmm_fields_out

  type, bind(c) :: lmm_stats
     integer(c_int) :: total_iter, outer_iter, vcycles, pressure_vcycles
     real(c_double) :: norm_b, norm_pre_b, norm_resid, norm_init_resid
     real(c_double) :: norm_resid_true, norm_init_true
     real(c_double) :: solve_ms, h2d_ms, d2h_ms
     integer(c_int) :: n_history
     real(c_double) :: history(LMM_HISTORY_MAX)
  end type lmm_stats

  interface

     subroutine lmm_default_knobs(k) bind(c, name="lmm_default_knobs")
       import :: lmm_knobs
       type(lmm_knobs), intent(out) :: k
     end subroutine lmm_default_knobs

     function lmm_stokes_create(g, k, device, h) bind(c, name="lmm_stokes_create") result(rc)
       import :: c_int, c_ptr, lmm_grid, lmm_knobs
       type(lmm_grid), intent(in) :: g
       type(lmm_knobs), intent(in) :: k
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: h
       integer(c_int) :: rc
     end function lmm_stokes_create

     function lmm_stokes_solve(h, fin, fout, theta_alpha, norm_pre_rhs, st) bind(c, name="lmm_stokes_solve") result(rc)
       import :: c_int, c_ptr, c_double, lmm_fields_in, lmm_fields_out, lmm_stats
       type(c_ptr), value :: h
       type(lmm_fields_in), intent(in) :: fin
       type(lmm_fields_out), intent(inout) :: fout
       real(c_double), intent(inout) :: theta_alpha
       real(c_double), intent(out) :: norm_pre_rhs
       type(lmm_stats), intent(out) :: st
       integer(c_int) :: rc
     end function lmm_stokes_solve

     function lmm_stokes_update_knobs(h, k) bind(c, name="lmm_stokes_update_knobs") result(rc)
       import :: c_int, c_ptr, lmm_knobs
       type(c_ptr), value :: h
       type(lmm_knobs), intent(in) :: k
       integer(c_int) :: rc
     end function lmm_stokes_update_knobs

     function lmm_stokes_destroy(h) bind(c, name="lmm_stokes_destroy") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int) :: rc
     end function lmm_stokes_destroy

     function lmm_strerror(code) bind(c, name="lmm_strerror") result(msg)
       import :: c_int, c_ptr
       integer(c_int), value :: code
       type(c_ptr) :: msg
     end function lmm_strerror

  end interface

contains

  ! the C message of a status code as a Fortran string
  function lmm_message(code) result(s)
    integer(c_int), intent(in) :: code
    character(len=256) :: s
    character(kind=c_char), pointer :: cs(:)
    integer :: i
    call c_f_pointer(lmm_strerror(code), cs, [256])
    s = ' '
    do i = 1, 256
       if (cs(i) == c_null_char) exit
       s(i:i) = cs(i)
    end do
  end function lmm_message

end module lmm_stokes_iface
