! gmres_lmm.f90 - drop-in replacement of src_gmres/gmres.f90.
!
! Same module name (gmres_module), same public subroutine and argument list
! as gmres.f90:30-45, so the time steppers (advance_timestep_overdamped.f90:
! 317,565; advance_timestep_inertial.f90:482,816) are unchanged.  The solve
! runs in liblmmstokes on the GPU: the multifab data of the single box are
! handed over with their ghost cells (LMM_LAYOUT_BOXLIB), the probin_gmres
! module globals are copied into lmm_knobs, and negative status codes end in
! bl_error exactly where the reference aborts.  One device handle is kept
! per grid and knob set and rebuilt when either changes.
!
! Restrictions of the library (checked at run time, status -1): one level,
! one box (max_grid_size >= n_cells); each direction periodic or bounded by
! walls on both sides (no-slip 100-103 or slip 200-203, from
! the_bc_tower%domain_bc); on a grid with walls, visc_schur_approx = 0 and no
! learned stage.
module gmres_module

  use iso_c_binding
  use multifab_module
  use ml_layout_module
  use define_bc_module
  use bl_error_module
  use probin_gmres_module
  use probin_common_module, only: visc_type
  use lmm_stokes_iface

  implicit none

  private
  public :: gmres

  type(c_ptr), save :: handle = c_null_ptr
  type(lmm_grid), save :: handle_grid
  type(lmm_knobs), save :: handle_knobs

contains

  subroutine gmres(mla,the_bc_tower,dx,b_u,b_p,x_u,x_p, &
                   alpha_fc,beta,beta_ed,gamma,theta_alpha,norm_pre_rhs)

    type(ml_layout),intent(in   ) :: mla
    type(bc_tower), intent(in   ) :: the_bc_tower
    real(dp_t)    , intent(in   ) :: dx(:,:)
    type(multifab), intent(inout) :: b_u(:,:)
    type(multifab), intent(in   ) :: b_p(:)
    type(multifab), intent(inout) :: x_u(:,:)
    type(multifab), intent(inout) :: x_p(:)
    type(multifab), intent(in   ) :: alpha_fc(:,:)
    type(multifab), intent(inout) :: beta(:)
    type(multifab), intent(inout) :: beta_ed(:,:)
    type(multifab), intent(inout) :: gamma(:)
    real(dp_t)    , intent(inout) :: theta_alpha
    real(dp_t), optional, intent(out) :: norm_pre_rhs

    type(lmm_grid) :: g
    type(lmm_knobs) :: k
    type(lmm_fields_in) :: fin
    type(lmm_fields_out) :: fout
    type(lmm_stats) :: st
    integer :: d, dm, lo(mla%dim), hi(mla%dim)
    integer(c_int) :: rc
    real(c_double) :: th, npr
    real(dp_t), pointer :: p(:,:,:,:)

    dm = mla%dim
    if (mla%nlevel .ne. 1) call bl_error("gmres: only one level is supported")
    if (nboxes(b_p(1)%la) .ne. 1) call bl_error("gmres: only one box is supported")

    lo = lwb(get_box(b_p(1),1))
    hi = upb(get_box(b_p(1),1))
    g%dm = dm
    g%n = 1
    g%n(1:dm) = hi - lo + 1
    g%dx = dx(1,1)
    ! physical BC codes per side (bc.f90: -1 periodic, 100-103 no-slip
    ! walls, 200-203 slip walls), as define_bc_tower received them
    g%bc_lo = LMM_BC_PERIODIC
    g%bc_hi = LMM_BC_PERIODIC
    do d = 1, dm
       if (.not. mla%pmask(d)) then
          g%bc_lo(d) = the_bc_tower%domain_bc(d,1)
          g%bc_hi(d) = the_bc_tower%domain_bc(d,2)
       end if
    end do

    call lmm_default_knobs(k)
    k%precon_type = precon_type
    k%visc_schur_approx = visc_schur_approx
    k%p_norm_weight = p_norm_weight
    k%scale_factor = scale_factor
    k%mg_verbose = mg_verbose
    k%cg_verbose = cg_verbose
    k%mg_max_vcycles = mg_max_vcycles
    k%mg_minwidth = mg_minwidth
    k%mg_bottom_solver = mg_bottom_solver
    k%mg_nsmooths_down = mg_nsmooths_down
    k%mg_nsmooths_up = mg_nsmooths_up
    k%mg_nsmooths_bottom = mg_nsmooths_bottom
    k%mg_max_bottom_nlevels = mg_max_bottom_nlevels
    k%mg_rel_tol = mg_rel_tol
    k%stag_mg_verbosity = stag_mg_verbosity
    k%stag_mg_max_vcycles = stag_mg_max_vcycles
    k%stag_mg_minwidth = stag_mg_minwidth
    k%stag_mg_bottom_solver = stag_mg_bottom_solver
    k%stag_mg_nsmooths_down = stag_mg_nsmooths_down
    k%stag_mg_nsmooths_up = stag_mg_nsmooths_up
    k%stag_mg_nsmooths_bottom = stag_mg_nsmooths_bottom
    k%stag_mg_max_bottom_nlevels = stag_mg_max_bottom_nlevels
    k%stag_mg_omega = stag_mg_omega
    k%stag_mg_smoother = stag_mg_smoother
    k%stag_mg_rel_tol = stag_mg_rel_tol
    k%gmres_rel_tol = gmres_rel_tol
    k%gmres_abs_tol = gmres_abs_tol
    k%gmres_verbose = gmres_verbose
    k%gmres_max_outer = gmres_max_outer
    k%gmres_max_inner = gmres_max_inner
    k%gmres_max_iter = gmres_max_iter
    k%gmres_min_iter = gmres_min_iter
    k%visc_type = visc_type

    if (c_associated(handle)) then
       if (.not. same_setup(g, k)) then
          rc = lmm_stokes_destroy(handle)
          handle = c_null_ptr
       else if (.not. same_stopping(k)) then
          ! the time steppers move gmres_abs_tol between predictor and
          ! corrector: keep the handle, change its stopping rules
          rc = lmm_stokes_update_knobs(handle, k)
          if (rc < 0) call bl_error("gmres: " // trim(lmm_message(rc)))
          handle_knobs = k
       end if
    end if
    if (.not. c_associated(handle)) then
       rc = lmm_stokes_create(g, k, 0_c_int, handle)
       if (rc < 0) call bl_error("gmres: " // trim(lmm_message(rc)))
       handle_grid = g
       handle_knobs = k
    end if

    ! the single fab of every multifab, ghost cells included
    fin%layout = LMM_LAYOUT_BOXLIB
    fin%b_u = c_null_ptr
    fin%alpha_fc = c_null_ptr
    fin%beta_ed = c_null_ptr
    do d = 1, dm
       p => dataptr(b_u(1,d), 1)
       fin%b_u(d) = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
       p => dataptr(alpha_fc(1,d), 1)
       fin%alpha_fc(d) = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    end do
    do d = 1, size(beta_ed,dim=2)
       p => dataptr(beta_ed(1,d), 1)
       fin%beta_ed(d) = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    end do
    p => dataptr(b_p(1), 1)
    fin%b_p = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    p => dataptr(beta(1), 1)
    fin%beta = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    p => dataptr(gamma(1), 1)
    fin%gamma = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    fin%ng_b_u = nghost(b_u(1,1))
    fin%ng_b_p = nghost(b_p(1))
    fin%ng_alpha = nghost(alpha_fc(1,1))
    fin%ng_beta = nghost(beta(1))
    fin%ng_beta_ed = nghost(beta_ed(1,1))
    fin%ng_gamma = nghost(gamma(1))

    fout%layout = LMM_LAYOUT_BOXLIB
    fout%x_u = c_null_ptr
    do d = 1, dm
       p => dataptr(x_u(1,d), 1)
       fout%x_u(d) = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    end do
    p => dataptr(x_p(1), 1)
    fout%x_p = c_loc(p(lbound(p,1),lbound(p,2),lbound(p,3),1))
    fout%ng_x_u = nghost(x_u(1,1))
    fout%ng_x_p = nghost(x_p(1))

    th = theta_alpha
    rc = lmm_stokes_solve(handle, fin, fout, th, npr, st)
    if (rc < 0) call bl_error("gmres.f90: " // trim(lmm_message(rc)))
    theta_alpha = th
    if (present(norm_pre_rhs)) norm_pre_rhs = npr

    if (gmres_verbose .ge. 1 .and. parallel_IOProcessor()) then
       if (rc > 0) write(*,*) 'gmres.f90: ', trim(lmm_message(rc))
       write(*,'(a)') 'Preconditioned GMRES:'
       write(*,'(a,i4)') '  total ITERs = ', st%total_iter
       write(*,'(a,100g17.9)') '  residual/(norm_b,initial) = ', st%norm_resid/st%norm_b, &
            st%norm_resid/st%norm_init_resid
    end if

  contains

    logical function same_setup(ga, ka)
      type(lmm_grid), intent(in) :: ga
      type(lmm_knobs), intent(in) :: ka
      same_setup = all(ga%n == handle_grid%n) .and. ga%dm == handle_grid%dm .and. ga%dx == handle_grid%dx &
           .and. ka%precon_type == handle_knobs%precon_type .and. ka%visc_type == handle_knobs%visc_type &
           .and. ka%gmres_max_inner == handle_knobs%gmres_max_inner .and. ka%method == handle_knobs%method &
           .and. ka%precision == handle_knobs%precision .and. ka%stag_mg_minwidth == handle_knobs%stag_mg_minwidth &
           .and. ka%mg_minwidth == handle_knobs%mg_minwidth &
           .and. ka%stag_mg_smoother == handle_knobs%stag_mg_smoother .and. ka%stag_mg_omega == handle_knobs%stag_mg_omega &
           .and. ka%stag_mg_nsmooths_down == handle_knobs%stag_mg_nsmooths_down &
           .and. ka%stag_mg_nsmooths_up == handle_knobs%stag_mg_nsmooths_up &
           .and. ka%stag_mg_nsmooths_bottom == handle_knobs%stag_mg_nsmooths_bottom &
           .and. ka%stag_mg_max_vcycles == handle_knobs%stag_mg_max_vcycles &
           .and. ka%mg_nsmooths_down == handle_knobs%mg_nsmooths_down .and. ka%mg_nsmooths_up == handle_knobs%mg_nsmooths_up &
           .and. ka%mg_nsmooths_bottom == handle_knobs%mg_nsmooths_bottom .and. ka%mg_max_vcycles == handle_knobs%mg_max_vcycles &
           .and. ka%p_norm_weight == handle_knobs%p_norm_weight &
           .and. ka%scale_factor == handle_knobs%scale_factor &
           .and. all(ga%bc_lo == handle_grid%bc_lo) .and. all(ga%bc_hi == handle_grid%bc_hi)
    end function same_setup

    ! the knobs lmm_stokes_update_knobs may change on a live handle
    logical function same_stopping(ka)
      type(lmm_knobs), intent(in) :: ka
      same_stopping = ka%gmres_rel_tol == handle_knobs%gmres_rel_tol .and. ka%gmres_abs_tol == handle_knobs%gmres_abs_tol &
           .and. ka%gmres_max_outer == handle_knobs%gmres_max_outer .and. ka%gmres_max_iter == handle_knobs%gmres_max_iter &
           .and. ka%gmres_min_iter == handle_knobs%gmres_min_iter .and. ka%mg_rel_tol == handle_knobs%mg_rel_tol &
           .and. ka%stag_mg_rel_tol == handle_knobs%stag_mg_rel_tol .and. ka%gmres_verbose == handle_knobs%gmres_verbose &
           .and. ka%mg_verbose == handle_knobs%mg_verbose .and. ka%cg_verbose == handle_knobs%cg_verbose &
           .and. ka%stag_mg_verbosity == handle_knobs%stag_mg_verbosity
    end function same_stopping

  end subroutine gmres

end module gmres_module
