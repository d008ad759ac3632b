! cfd_b200_mod.f90 - Fortran 2003 (iso_c_binding) interfaces to the C ABI of cfd_b200.h.
!
! For the reference's Fortran driver (littleharsh.f90): add this file next to
! declaration.f90, `use cfd_b200_mod`, and link with -L<repo>/cfd_b200/_lib -lcfdb200.
! Every function of cfd_b200.h has an interface here with the same name and arguments:
! C scalars passed by value carry `value`, C pointers to host data are assumed-size
! arrays or scalars passed by reference, and device pointers, streams and opaque handles
! are type(c_ptr), value (handles returned through a pointer are type(c_ptr), intent(out)).
! Spectral host fields are the reference's complex(8) cfield%f(j,column) arrays.
module cfd_b200_mod
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: CFD_OK = 0, CFD_ERR_ARG = 1, CFD_ERR_SIZE = 2, CFD_ERR_CUDA = 3
  integer(c_int), parameter :: CFD_ERR_NONFINITE = 4, CFD_ERR_STATE = 5, CFD_ERR_NOMEM = 6
  integer(c_int32_t), parameter :: CFD_PREC_FP64 = 0, CFD_PREC_MIXED = 1
  integer(c_int32_t), parameter :: CFD_FIELD_U1 = 0, CFD_FIELD_U2 = 1, CFD_FIELD_U3 = 2, CFD_FIELD_P = 3
  integer(c_int32_t), parameter :: CFD_FIELD_NU1 = 4, CFD_FIELD_NU2 = 5, CFD_FIELD_NU3 = 6
  integer(c_int32_t), parameter :: CFD_FIELD_DIV = 7, CFD_FIELD_PSI = 8
  integer(c_int32_t), parameter :: CFD_FIELD_DU1 = 9, CFD_FIELD_DU2 = 10, CFD_FIELD_DU3 = 11
  integer(c_int32_t), parameter :: CFD_LAYOUT_REF = 0, CFD_LAYOUT_PLANE = 1

  type, bind(c) :: cfd_config
    integer(c_int32_t) :: ngal1, ngal2, ny, dsty
    real(c_double)     :: re, alp, bet, dt, mpgx, qxt
    integer(c_int32_t) :: flag_ctpress, precision
    type(c_ptr)        :: yu, yv, dthdyu, dthdyv, dyu2i, dyv2i
    integer(c_int32_t) :: ngal1_mid, ngal2_mid, band_vface
  end type

  type, bind(c) :: cfd_ib_list
    integer(c_int32_t) :: n
    type(c_ptr)        :: idx, w
    integer(c_int32_t) :: jlo(2), jhi(2)
  end type

  type, bind(c) :: cfd_tuning
    integer(c_int32_t) :: xline_path, xline_rows, zlines, solve_kind, solve_cols, rhs_chunk, xsplit, zsplit
  end type

  type, bind(c) :: cfd_stats_config
    integer(c_int32_t) :: jband, dnx, dnz, spectra
  end type

  interface
    ! ---- context -----------------------------------------------------------------------
    integer(c_int) function cfd_create(cfg, ibu, ibv, device, ctx) bind(c, name='cfd_create')
      import; type(cfd_config), intent(in) :: cfg; type(cfd_ib_list), intent(in) :: ibu, ibv
      integer(c_int32_t), value :: device; type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function cfd_create_tuned(cfg, ibu, ibv, device, tuning, ctx) bind(c, name='cfd_create_tuned')
      import; type(cfd_config), intent(in) :: cfg; type(cfd_ib_list), intent(in) :: ibu, ibv
      integer(c_int32_t), value :: device; type(cfd_tuning), intent(in) :: tuning
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function cfd_destroy(ctx) bind(c, name='cfd_destroy')
      import; type(c_ptr), value :: ctx
    end function
    type(c_ptr) function cfd_last_error(ctx) bind(c, name='cfd_last_error')
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function cfd_get_tuning(ctx, tuning) bind(c, name='cfd_get_tuning')
      import; type(c_ptr), value :: ctx; type(cfd_tuning), intent(out) :: tuning
    end function
    integer(c_int) function cfd_set_stream(ctx, stream) bind(c, name='cfd_set_stream')
      import; type(c_ptr), value :: ctx, stream
    end function
    integer(c_int) function cfd_synchronize(ctx) bind(c, name='cfd_synchronize')
      import; type(c_ptr), value :: ctx
    end function

    ! ---- fields --------------------------------------------------------------------------
    integer(c_int) function cfd_field_shape(ctx, field, ncomplex, j0, nplanes, ncolumns) bind(c, name='cfd_field_shape')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: field
      integer(c_int64_t), intent(out) :: ncomplex; integer(c_int32_t), intent(out) :: j0, nplanes, ncolumns
    end function
    integer(c_int) function cfd_upload_field(ctx, field, host, layout) bind(c, name='cfd_upload_field')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: field, layout
      complex(c_double_complex), intent(in) :: host(*)
    end function
    integer(c_int) function cfd_download_field(ctx, field, host, layout) bind(c, name='cfd_download_field')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: field, layout
      complex(c_double_complex), intent(out) :: host(*)
    end function
    integer(c_int) function cfd_field_device_ptr(ctx, field, dev_ptr) bind(c, name='cfd_field_device_ptr')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: field
      type(c_ptr), intent(out) :: dev_ptr
    end function

    ! ---- stages of one RK3 substep (littleharsh.f90:163-189) and whole steps -------------
    integer(c_int) function cfd_rhs0(ctx, krk) bind(c, name='cfd_rhs0')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_nonlinear(ctx, krk) bind(c, name='cfd_nonlinear')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_solve_uvw(ctx, krk) bind(c, name='cfd_solve_uvw')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_meanflow(ctx, krk) bind(c, name='cfd_meanflow')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_solve_p(ctx, krk) bind(c, name='cfd_solve_p')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_vcorr(ctx, krk) bind(c, name='cfd_vcorr')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_rk_substep(ctx, krk) bind(c, name='cfd_rk_substep')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: krk
    end function
    integer(c_int) function cfd_step(ctx, nsteps) bind(c, name='cfd_step')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: nsteps
    end function
    integer(c_int) function cfd_get_scalars(ctx, mpgx, qx, dgx) bind(c, name='cfd_get_scalars')
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: mpgx, qx, dgx
    end function
    integer(c_int) function cfd_divergence_max(ctx, errmax) bind(c, name='cfd_divergence_max')
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: errmax
    end function

    ! ---- transforms on device planes (four_to_phys_du, phys_to_four_du, rft, cft) ----------
    integer(c_int) function cfd_four_to_phys(ctx, planes, nplanes, zero_oddball) bind(c, name='cfd_four_to_phys')
      import; type(c_ptr), value :: ctx, planes; integer(c_int32_t), value :: nplanes, zero_oddball
    end function
    integer(c_int) function cfd_phys_to_four(ctx, planes, nplanes) bind(c, name='cfd_phys_to_four')
      import; type(c_ptr), value :: ctx, planes; integer(c_int32_t), value :: nplanes
    end function
    integer(c_int) function cfd_rft(ctx, cvec, isa, m, iopt) bind(c, name='cfd_rft')
      import; type(c_ptr), value :: ctx, cvec; integer(c_int32_t), value :: isa, m, iopt
    end function
    integer(c_int) function cfd_cft(ctx, cvec, ise, isa, m, iopt) bind(c, name='cfd_cft')
      import; type(c_ptr), value :: ctx, cvec; integer(c_int32_t), value :: ise, isa, m, iopt
    end function

    ! ---- statistics, spectra and CFL (stats.f90, spectra.f90, dtc_calc) --------------------
    integer(c_int) function cfd_stats_configure(ctx, sc) bind(c, name='cfd_stats_configure')
      import; type(c_ptr), value :: ctx; type(cfd_stats_config), intent(in) :: sc
    end function
    integer(c_int) function cfd_stats_accumulate(ctx) bind(c, name='cfd_stats_accumulate')
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function cfd_stats_reset(ctx) bind(c, name='cfd_stats_reset')
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function cfd_stats_read(ctx, su, sv, sp, cu, cv, cp, istat) bind(c, name='cfd_stats_read')
      import; type(c_ptr), value :: ctx
      real(c_double), intent(out) :: su(*), sv(*), sp(*), cu(*), cv(*), cp(*)
      integer(c_int32_t), intent(out) :: istat
    end function
    integer(c_int) function cfd_spectra_read(ctx, spu, spv, spw, spuv, spp) bind(c, name='cfd_spectra_read')
      import; type(c_ptr), value :: ctx
      real(c_double), intent(out) :: spu(*), spv(*), spw(*), spuv(*), spp(*)
    end function
    integer(c_int) function cfd_cfl(ctx, dtc, terms) bind(c, name='cfd_cfl')
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: dtc, terms(3)
    end function
    integer(c_int) function cfd_set_dt(ctx, dt) bind(c, name='cfd_set_dt')
      import; type(c_ptr), value :: ctx; real(c_double), value :: dt
    end function
    integer(c_int) function cfd_set_lastplane(ctx, on) bind(c, name='cfd_set_lastplane')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: on
    end function

    ! ---- ensembles ----------------------------------------------------------------------------
    integer(c_int) function cfd_ensemble_create(members, nmembers, ens) bind(c, name='cfd_ensemble_create')
      import; type(c_ptr), intent(in) :: members(*); integer(c_int32_t), value :: nmembers
      type(c_ptr), intent(out) :: ens
    end function
    integer(c_int) function cfd_ensemble_step(ens, nsteps) bind(c, name='cfd_ensemble_step')
      import; type(c_ptr), value :: ens; integer(c_int32_t), value :: nsteps
    end function
    integer(c_int) function cfd_ensemble_synchronize(ens) bind(c, name='cfd_ensemble_synchronize')
      import; type(c_ptr), value :: ens
    end function
    integer(c_int) function cfd_ensemble_stream(ens, stream) bind(c, name='cfd_ensemble_stream')
      import; type(c_ptr), value :: ens; type(c_ptr), intent(out) :: stream
    end function
    type(c_ptr) function cfd_ensemble_last_error(ens) bind(c, name='cfd_ensemble_last_error')
      import; type(c_ptr), value :: ens
    end function
    integer(c_int) function cfd_ensemble_destroy(ens) bind(c, name='cfd_ensemble_destroy')
      import; type(c_ptr), value :: ens
    end function

    ! ---- LUsolU on caller-owned device memory, no context ------------------------------------
    integer(c_int) function cfd_lusol_u_noalloc(nkx, n2, nplanes, beta, gw_bot, gw_top, kx, kz, dyu2i, rhs, u, &
                                                stream) bind(c, name='cfd_lusol_u_noalloc')
      import; integer(c_int32_t), value :: nkx, n2, nplanes; real(c_double), value :: beta, gw_bot, gw_top
      type(c_ptr), value :: kx, kz, dyu2i, rhs, u, stream
    end function

    ! ---- diagnostics ----------------------------------------------------------------------
    integer(c_int) function cfd_profile(ctx, enable) bind(c, name='cfd_profile')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: enable
    end function
    integer(c_int) function cfd_profile_read(ctx, buf, buflen) bind(c, name='cfd_profile_read')
      import; type(c_ptr), value :: ctx; character(kind=c_char), intent(out) :: buf(*)
      integer(c_int32_t), value :: buflen
    end function
    integer(c_int) function cfd_launch_count(ctx, count) bind(c, name='cfd_launch_count')
      import; type(c_ptr), value :: ctx; integer(c_int64_t), intent(out) :: count
    end function
    type(c_ptr) function cfd_version() bind(c, name='cfd_version')
      import
    end function
  end interface
end module cfd_b200_mod
