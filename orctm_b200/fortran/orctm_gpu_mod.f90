! ISO_C_BINDING interface to liborctm_gpu.so (include/orctm_gpu.h) for the
! ORCTM Fortran host.  The reference's subroutines keep their names; their
! bodies become calls of the entry points below (OCVTOT_NH calls
! orctm_ocvtot_nh, petsc_start orctm_create, ...).  Compile with the model
! (-fdefault-real-8 / -r8 as the model itself) and link -lorctm_gpu -lcudart.
module orctm_gpu_mod
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: ORCTM_OK = 0, ORCTM_E_NOT_CONVERGED = -4
  integer(c_int), parameter :: ORCTM_F_UOO = 0, ORCTM_F_VOE = 1, ORCTM_F_WNO = 2, &
       ORCTM_F_UKO = 3, ORCTM_F_VKE = 4, ORCTM_F_WO = 5, ORCTM_F_UOO_1 = 6, &
       ORCTM_F_VOE_1 = 7, ORCTM_F_WNO_1 = 8, ORCTM_F_PNH = 9, ORCTM_F_ZO = 10, &
       ORCTM_F_DVO = 11, ORCTM_F_AVO = 12, ORCTM_F_THO = 13, ORCTM_F_SAO = 14
  integer(c_int), parameter :: ORCTM_E_UNSTABLE = -9
  integer(c_int), parameter :: ORCTM_EOS_UNESCO = 0, ORCTM_EOS_LINEAR = 1
  integer(c_int), parameter :: ORCTM_C_PO = 0, ORCTM_C_STABIO = 1, ORCTM_C_RHOO = 2, &
       ORCTM_C_UK1O = 3, ORCTM_C_VK1E = 4, ORCTM_C_EMINPO = 5, ORCTM_C_RIVRUN = 6, &
       ORCTM_C_KCONDEP = 7

  type, bind(c) :: orctm_desc
     integer(c_int) :: ie, je, ke, i_start, j_start, ntracers
     integer(c_int) :: ob_west, ob_east, ob_north, ob_south
     real(c_double) :: dt, almzer, aulapts, aulapuv, ah00
     type(c_ptr) :: dzw, di
     type(c_ptr) :: dlxp, dlyp, dtdxpo, dtdyo
     type(c_ptr) :: dlxu, dlyu, dtdxuo
     type(c_ptr) :: dlxv, dlyv, dpye
     type(c_ptr) :: ddpo, weto, dduo, amsuo, ddue, amsue
     integer(c_int) :: device
  end type orctm_desc

  type, bind(c) :: orctm_solve_stats
     integer(c_int) :: iterations, outer_iterations, converged
     real(c_double) :: relres, relres_initial, solve_ms
  end type orctm_solve_stats

  ! coordinates and depths of GRID_INFO.ext (orctm_write_gridinfo)
  type, bind(c) :: orctm_gridinfo
     type(c_ptr) :: lonp, latp, lonu, latu, lonv, latv, depto, deuto, deute
  end type orctm_gridinfo

  ! open-boundary tidal constants and sponge parameters; amp(v, s), pha(v, s)
  ! with v = 1..3 (z, u, v) and s = 1..4 (west, east, north, south)
  type, bind(c) :: orctm_obc
     integer(c_int) :: ntide
     type(c_ptr) :: period
     integer(c_int) :: sponge(4), width(4)
     real(c_double) :: relax_inner, relax_bound
     type(c_ptr) :: amp(3, 4), pha(3, 4)
  end type orctm_obc

  ! barotropic solve (ITPREP's inputs and the run's constants)
  type, bind(c) :: orctm_barotropic
     type(c_ptr) :: deuto, deute
     real(c_double) :: minvalue, grav, stabn, conn, rlsa1, sorpar
     integer(c_int) :: niter, eta_forc
  end type orctm_barotropic

  ! OCTHER's constants and surface forcing (orctm.f90:311-330, 503, 561-569, 739-743)
  type, bind(c) :: orctm_thermo
     integer(c_int) :: eos
     real(c_double) :: rho0, drdt, drds, t0, s0
     real(c_double) :: grav
     real(c_double) :: relsal, reltem
     real(c_double) :: rhoicwa, rhosnwa
     real(c_double) :: wt
     real(c_double) :: cstabeps, dv0, av0, cavocon, cdvocon
     type(c_ptr) :: preff
     type(c_ptr) :: dbackv
     type(c_ptr) :: abackv
     type(c_ptr) :: sicomo, sictho, sicsno
     type(c_ptr) :: relsao, reltho
     type(c_ptr) :: giriv
     type(c_ptr) :: fu10
  end type orctm_thermo

  ! OCMODMOM's Coriolis inputs (the grid file's FTWOU, FTWOV; coriol.f90's GILA, GIPH)
  type, bind(c) :: orctm_coriolis
     type(c_ptr) :: ftwou, ftwov, gila, giph
     real(c_double) :: omega
  end type orctm_coriolis

  interface
     integer(c_int) function orctm_create(desc, h) bind(c, name="orctm_create")
       import :: c_int, c_ptr, orctm_desc
       type(orctm_desc), intent(in) :: desc
       type(c_ptr), intent(out) :: h
     end function
     integer(c_int) function orctm_destroy(h) bind(c, name="orctm_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_upload(h, field, host, n) bind(c, name="orctm_upload")
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: h
       integer(c_int), value :: field
       type(c_ptr), value :: host
       integer(c_size_t), value :: n
     end function
     integer(c_int) function orctm_download(h, field, host, n) bind(c, name="orctm_download")
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: h
       integer(c_int), value :: field
       type(c_ptr), value :: host
       integer(c_size_t), value :: n
     end function
     integer(c_int) function orctm_ocuad(h) bind(c, name="orctm_ocuad")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocvad(h) bind(c, name="orctm_ocvad")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocwad(h) bind(c, name="orctm_ocwad")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocadpo(h, tracer) bind(c, name="orctm_ocadpo")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: tracer
     end function
     integer(c_int) function orctm_octdiff(h) bind(c, name="orctm_octdiff")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_octimf(h) bind(c, name="orctm_octimf")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_set_obc(h, obc) bind(c, name="orctm_set_obc")
       import :: c_int, c_ptr, orctm_obc
       type(c_ptr), value :: h
       type(orctm_obc), intent(in) :: obc
     end function
     integer(c_int) function orctm_obc_eta(h, ldtrun) bind(c, name="orctm_obc_eta")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: ldtrun
     end function
     integer(c_int) function orctm_obc_uv(h, ldtrun) bind(c, name="orctm_obc_uv")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: ldtrun
     end function
     ! cli(s): c_loc of side s's climatology record (n, KE), c_null_ptr if unused
     integer(c_int) function orctm_set_obc_ts(h, tracer, cli) bind(c, name="orctm_set_obc_ts")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: tracer
       type(c_ptr), dimension(4), intent(in) :: cli
     end function
     integer(c_int) function orctm_obc_ts(h) bind(c, name="orctm_obc_ts")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     ! OBC_SPONGE_EXP with the namelist TAO (s); 0 returns to the 1/x sponge
     integer(c_int) function orctm_set_obc_sponge_exp(h, tao) bind(c, name="orctm_set_obc_sponge_exp")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: tao
     end function
     integer(c_int) function orctm_set_barotropic(h, b) bind(c, name="orctm_set_barotropic")
       import :: c_int, c_ptr, orctm_barotropic
       type(c_ptr), value :: h
       type(orctm_barotropic), intent(in) :: b
     end function
     integer(c_int) function orctm_troneu(h, u1o, v1e, uzo, vze) bind(c, name="orctm_troneu")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, u1o, v1e, uzo, vze
     end function
     integer(c_int) function orctm_ocvtro(h) bind(c, name="orctm_ocvtro")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocvtot(h) bind(c, name="orctm_ocvtot")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_trotest(h, ntry, niter, sorpar) bind(c, name="orctm_trotest")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: ntry, niter
       real(c_double), intent(out) :: sorpar
     end function
     integer(c_int) function orctm_ocbarp(h) bind(c, name="orctm_ocbarp")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocwind(h, txo, tye, sicomu, sicomv, tauwatu, tauwatv) &
         bind(c, name="orctm_ocwind")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, txo, tye, sicomu, sicomv, tauwatu, tauwatv
     end function
     integer(c_int) function orctm_set_thermo(h, t) bind(c, name="orctm_set_thermo")
       import :: c_int, c_ptr, orctm_thermo
       type(c_ptr), value :: h
       type(orctm_thermo), intent(in) :: t
     end function
     integer(c_int) function orctm_set_coriolis(h, c) bind(c, name="orctm_set_coriolis")
       import :: c_int, c_ptr, orctm_coriolis
       type(c_ptr), value :: h
       type(orctm_coriolis), intent(in) :: c
     end function
     integer(c_int) function orctm_octher(h) bind(c, name="orctm_octher")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocmodmom(h) bind(c, name="orctm_ocmodmom")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_occlit(h, contra) bind(c, name="orctm_occlit")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: contra
     end function
     integer(c_int) function orctm_upload_baroclinic(h, which, host, n) &
         bind(c, name="orctm_upload_baroclinic")
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: h, host
       integer(c_int), value :: which
       integer(c_size_t), value :: n
     end function
     integer(c_int) function orctm_download_baroclinic(h, which, host, n) &
         bind(c, name="orctm_download_baroclinic")
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: h, host
       integer(c_int), value :: which
       integer(c_size_t), value :: n
     end function
     integer(c_int) function orctm_step_full(h, ldtrun, stats, contra) bind(c, name="orctm_step_full")
       import :: c_int, c_ptr, c_double, orctm_solve_stats
       type(c_ptr), value :: h
       integer(c_int), value :: ldtrun
       type(orctm_solve_stats), intent(out) :: stats
       real(c_double), intent(out) :: contra
     end function
     integer(c_int) function orctm_download_barotropic(h, which, host, n) &
         bind(c, name="orctm_download_barotropic")
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: h, host
       integer(c_int), value :: which
       integer(c_size_t), value :: n
     end function
     integer(c_int) function orctm_ocvisc(h) bind(c, name="orctm_ocvisc")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_ocvtot_nh(h, stats) bind(c, name="orctm_ocvtot_nh")
       import :: c_int, c_ptr, orctm_solve_stats
       type(c_ptr), value :: h
       type(orctm_solve_stats), intent(out) :: stats
     end function
     integer(c_int) function orctm_ocadpo_all(h) bind(c, name="orctm_ocadpo_all")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function orctm_step_hotpath(h, stats) bind(c, name="orctm_step_hotpath")
       import :: c_int, c_ptr, orctm_solve_stats
       type(c_ptr), value :: h
       type(orctm_solve_stats), intent(out) :: stats
     end function
     integer(c_int) function orctm_synchronize(h) bind(c, name="orctm_synchronize")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     ! path: a NUL-terminated string, e.g. 'fort.71'//c_null_char
     integer(c_int) function orctm_write_extra(h, path, append, idate, nfield, fields, codes) &
         bind(c, name="orctm_write_extra")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*), intent(in) :: path
       integer(c_int), value :: append, idate, nfield
       integer(c_int), dimension(*), intent(in) :: fields, codes
     end function
     integer(c_int) function orctm_read_extra(h, path, nfield, fields, codes) &
         bind(c, name="orctm_read_extra")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*), intent(in) :: path
       integer(c_int), value :: nfield
       integer(c_int), dimension(*), intent(in) :: fields, codes
     end function
     integer(c_int) function orctm_write_gridinfo(path, desc, g) bind(c, name="orctm_write_gridinfo")
       import :: c_int, c_char, orctm_desc, orctm_gridinfo
       character(kind=c_char), dimension(*), intent(in) :: path
       type(orctm_desc), intent(in) :: desc
       type(orctm_gridinfo), intent(in) :: g
     end function
     integer(c_int) function orctm_set_solver(h, mode, rtol, maxit) bind(c, name="orctm_set_solver")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: mode, maxit
       real(c_double), value :: rtol
     end function
     integer(c_int) function orctm_set_tuning(h, col_variant, spmv_variant) &
         bind(c, name="orctm_set_tuning")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: col_variant, spmv_variant
     end function
     integer(c_int) function orctm_device_bytes(h, bytes) bind(c, name="orctm_device_bytes")
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: h
       integer(c_long_long), intent(out) :: bytes
     end function
     integer(c_int) function orctm_trim_device_memory(device) &
         bind(c, name="orctm_trim_device_memory")
       import :: c_int
       integer(c_int), value :: device
     end function
  end interface

  type(c_ptr), save :: orctm_h = c_null_ptr
end module orctm_gpu_mod
