!> wa_module_b200 -- ISO_C_BINDING front end of libdogcm_sht.so for dogcm.
!!
!! It exports the SPMODEL wa_module names that SpmlUtil_mod re-exports
!! (SpmlUtil_mod.f90:105-135), with the same dummy shapes, and routes every
!! horizontal transform to the B200 library through the C-ABI of
!! include/dogcm_sht.h.  It also exports fused forms of SpmlUtil_mod's
!! composites (w_AlphaOptr_xy, calc_VorDiv2UV, ...) that take one library
!! call instead of two to four SPMODEL calls.  Swap `use wa_module`
!! (SpmlUtil_mod.f90:41-46) for `use wa_module_b200` to adopt it.
!!
!! Errors: every C entry point returns a status; a nonzero one is reported with
!! MessageNotify('E', ...), which aborts, as the reference does on misuse.
module wa_module_b200

  use iso_c_binding
  use dc_types, only: DP
  use dc_message, only: MessageNotify

  implicit none
  private

  public :: wa_Initial, wa_Finalize, b200_SetPrecision
  public :: x_Lon, y_Lat, x_Lon_Weight, y_Lat_Weight, xy_Lon, xy_Lat
  public :: rn, l_nm, nm_l
  public :: w_xy, xy_w, wa_xya, xya_wa
  public :: w_DivLambda_xy, w_DivMu_xy
  public :: xy_GradLambda_w, xy_GradMu_w, xy_GradLon_w, xy_GradLat_w
  public :: xya_GradLambda_wa, xya_GradMu_wa, xya_GradLon_wa, xya_GradLat_wa
  public :: w_Lapla_w, w_LaplaInv_w
  public :: AvrLonLat_xy, IntLonLat_xy, ya_AvrLon_xya, ya_IntLon_xya
  public :: b200_wa_AlphaOptr_xya, b200_xya_AlphaOptr_wa
  public :: b200_calc_UVCosLat2VorDiv, b200_calc_VorDiv2UV, b200_calc_MomProd2VorDiv
  public :: b200_wa_Diffuse
  public :: b200_wa_AlphaOptrProd_xya, b200_xya_HGrad_wa, b200_xya_HGrad_xya, b200_xya_FluxDiv_xya
  public :: b200_wa_xyz_section, b200_xyz_wa_section
  ! legacy spellings of the horizontal transforms of the sogcm SpmlUtil_mod
  ! (model/old/sogcm/util/SpmlUtil_mod.f90:75-84,308-344,529-679)
  public :: xyz_wz, wz_xyz, wt_xyt
  public :: wz_AlphaOptr_xyz, xyz_AlphaOptr_wz
  public :: w_Lapla2D_w, wz_Lapla2D_wz, w_InvLapla2D_w, wz_InvLapla2D_wz

  integer, parameter :: SHT_OK = 0
  ! precision modes of the Legendre contraction (include/dogcm_sht.h)
  integer, parameter, public :: SHT_PREC_FP64 = 0, SHT_PREC_SPLIT = 1, SHT_PREC_AUTO = 2
  character(*), parameter :: module_name = 'wa_module_b200'

  type(c_ptr), save :: plan = c_null_ptr
  integer, save :: im = 0, jm = 0, nm = 0, lm = 0
  real(DP), save :: radius_ = 1.0_DP   ! planetary radius given to wa_Initial

  real(DP), save, allocatable :: x_Lon(:), y_Lat(:), x_Lon_Weight(:), y_Lat_Weight(:)
  real(DP), save, allocatable :: xy_Lon(:,:), xy_Lat(:,:)
  real(DP), save, allocatable :: rn(:,:)

  interface
    integer(c_int) function sht_init(im, jm, km, nm, radius, plan) bind(C, name='sht_init')
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: im, jm, km, nm
      real(c_double), value :: radius
      type(c_ptr), intent(out) :: plan
    end function sht_init
    integer(c_int) function sht_final(plan) bind(C, name='sht_final')
      import :: c_int, c_ptr
      type(c_ptr), value :: plan
    end function sht_final
    integer(c_int) function sht_dims(plan, im, jm, nm, lm) bind(C, name='sht_dims')
      import :: c_int, c_ptr
      type(c_ptr), value :: plan
      integer(c_int), intent(out) :: im, jm, nm, lm
    end function sht_dims
    integer(c_int) function sht_grid_info(plan, x_lon, y_lat, x_w, y_w) bind(C, name='sht_grid_info')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan
      real(c_double), intent(out) :: x_lon(*), y_lat(*), x_w(*), y_w(*)
    end function sht_grid_info
    integer(c_int) function sht_set_precision(plan, mode) bind(C, name='sht_set_precision')
      import :: c_int, c_ptr
      type(c_ptr), value :: plan
      integer(c_int), value :: mode
    end function sht_set_precision
    integer(c_int) function sht_rn(plan, rnv) bind(C, name='sht_rn')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan
      real(c_double), intent(out) :: rnv(*)
    end function sht_rn
    function sht_last_error() bind(C, name='sht_last_error')
      import :: c_ptr
      type(c_ptr) :: sht_last_error
    end function sht_last_error
  end interface

  ! One interface per entry point (each is a distinct C symbol).
  interface
    integer(c_int) function sht_wa_xya(plan, x, nb, w) bind(C, name='sht_wa_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_wa(plan, x, nb, w) bind(C, name='sht_xya_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_wa_divlambda_xya(plan, x, nb, w) bind(C, name='sht_wa_divlambda_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_wa_divmu_xya(plan, x, nb, w) bind(C, name='sht_wa_divmu_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_gradlambda_wa(plan, x, nb, w) bind(C, name='sht_xya_gradlambda_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_gradmu_wa(plan, x, nb, w) bind(C, name='sht_xya_gradmu_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_gradlon_wa(plan, x, nb, w) bind(C, name='sht_xya_gradlon_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_gradlat_wa(plan, x, nb, w) bind(C, name='sht_xya_gradlat_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_wa_lapla_wa(plan, x, nb, w) bind(C, name='sht_wa_lapla_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_wa_laplainv_wa(plan, x, nb, w) bind(C, name='sht_wa_laplainv_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_avrlonlat_xya(plan, x, nb, w) bind(C, name='sht_avrlonlat_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_intlonlat_xya(plan, x, nb, w) bind(C, name='sht_intlonlat_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_ya_avrlon_xya(plan, x, nb, w) bind(C, name='sht_ya_avrlon_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_ya_intlon_xya(plan, x, nb, w) bind(C, name='sht_ya_intlon_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_wa_alphaoptr_xya(plan, a, b, nb, w) bind(C, name='sht_wa_alphaoptr_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: a(*), b(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_xya_alphaoptr_wa(plan, a, b, nb, x) bind(C, name='sht_xya_alphaoptr_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: a(*), b(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: x(*)
    end function
    integer(c_int) function sht_uvcoslat2vordiv(plan, u, v, nb, vor, div) bind(C, name='sht_uvcoslat2vordiv')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: u(*), v(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: vor(*), div(*)
    end function
    integer(c_int) function sht_vordiv2uv(plan, vor, div, nb, u, v) bind(C, name='sht_vordiv2uv')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: vor(*), div(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: u(*), v(*)
    end function
    integer(c_int) function sht_wa_alphaoptr_prod_xya(plan, a, b, q, nb, w) bind(C, name='sht_wa_alphaoptr_prod_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: a(*), b(*), q(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: w(*)
    end function
    integer(c_int) function sht_uvcoslat2vordiv_fma(plan, x1, x2, q, z1, z2, nb, vor, div) &
         bind(C, name='sht_uvcoslat2vordiv_fma')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x1(*), x2(*), q(*), z1(*), z2(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: vor(*), div(*)
    end function
    integer(c_int) function sht_xya_hgrad_wa(plan, w, nb, glon, glat) bind(C, name='sht_xya_hgrad_wa')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: w(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: glon(*), glat(*)
    end function
    integer(c_int) function sht_xya_hgrad_xya(plan, x, nb, glon, glat) bind(C, name='sht_xya_hgrad_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: x(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: glon(*), glat(*)
    end function
    integer(c_int) function sht_xya_fluxdiv_xya(plan, a, b, nb, x) bind(C, name='sht_xya_fluxdiv_xya')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(in) :: a(*), b(*)
      integer(c_int), value :: nb; real(c_double), intent(out) :: x(*)
    end function
    integer(c_int) function sht_analysis(plan, x, ldi, ldj, nb, w, ldw, mode) bind(C, name='sht_analysis')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan, x
      integer(c_int), value :: ldi, ldj, nb
      real(c_double), intent(out) :: w(*)
      integer(c_int), value :: ldw, mode
    end function
    integer(c_int) function sht_synthesis(plan, w, ldw, nb, x, ldi, ldj, mode) bind(C, name='sht_synthesis')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan
      real(c_double), intent(in) :: w(*)
      integer(c_int), value :: ldw, nb
      type(c_ptr), value :: x
      integer(c_int), value :: ldi, ldj, mode
    end function
    integer(c_int) function sht_wa_diffuse(plan, w, nb, coef, dt, filt) bind(C, name='sht_wa_diffuse')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: plan; real(c_double), intent(inout) :: w(*)
      integer(c_int), value :: nb; real(c_double), intent(in) :: coef(*)
      real(c_double), value :: dt; real(c_double), intent(in) :: filt(*)
    end function
  end interface

contains

  subroutine check(status, where)
    integer(c_int), intent(in) :: status
    character(*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    character(len=256) :: text
    integer :: k
    if (status == SHT_OK) return
    call c_f_pointer(sht_last_error(), msg, [256])
    text = ''
    do k = 1, 256
       if (msg(k) == c_null_char) exit
       text(k:k) = msg(k)
    end do
    call MessageNotify('E', module_name, trim(where)//': '//trim(text))
  end subroutine check

  !> wa_Initial(nm, im, jm, km[, np]) of SPMODEL (SpmlUtil_mod.f90:218-223); radius
  !! is the planetary radius used by the fused composites (1 = unit sphere).
  !! np (the SPMODEL OpenMP thread count) has no meaning on the GPU and is ignored.
  subroutine wa_Initial(n_in, i_in, j_in, k_in, np, radius)
    integer, intent(in) :: n_in, i_in, j_in, k_in
    integer, intent(in), optional :: np
    real(DP), intent(in), optional :: radius
    real(DP) :: a
    integer :: i, j
    integer(c_int) :: ci, cj, cn, cl
    a = 1.0_DP
    if (present(radius)) a = radius
    radius_ = a
    call check(sht_init(int(i_in, c_int), int(j_in, c_int), int(k_in, c_int), int(n_in, c_int), &
         real(a, c_double), plan), 'wa_Initial')
    ! the plan fixes nm (nm = -1 selects the default) and lm: (nm+1)**2, or
    ! nm+1 for the axisymmetric model (im = 1, SpmlUtil_mod.f90:210-214)
    call check(sht_dims(plan, ci, cj, cn, cl), 'wa_Initial')
    im = ci; jm = cj; nm = cn; lm = cl
    allocate(x_Lon(0:im-1), y_Lat(jm), x_Lon_Weight(0:im-1), y_Lat_Weight(jm))
    allocate(xy_Lon(0:im-1, jm), xy_Lat(0:im-1, jm), rn(lm, 2))
    call check(sht_grid_info(plan, x_Lon, y_Lat, x_Lon_Weight, y_Lat_Weight), 'wa_Initial')
    do j = 1, jm
       do i = 0, im-1
          xy_Lon(i, j) = x_Lon(i); xy_Lat(i, j) = y_Lat(j)
       end do
    end do
    call check(sht_rn(plan, rn(:, 1)), 'wa_Initial')
    rn(:, 2) = 0.0_DP  ! only rn(:,1), the Laplacian eigenvalue, is used by dogcm
  end subroutine wa_Initial

  !> Precision of the following transforms: SHT_PREC_FP64 (the default),
  !> SHT_PREC_SPLIT (integer digit products on the tensor cores, <= 1e-11
  !> relative) or SHT_PREC_AUTO (split where a contraction has at least 128
  !> terms: the faster of the two per direction).  No counterpart in SPMODEL.
  subroutine b200_SetPrecision(mode)
    integer, intent(in) :: mode
    call check(sht_set_precision(plan, int(mode, c_int)), 'SetPrecision')
  end subroutine b200_SetPrecision

  subroutine wa_Finalize()
    if (c_associated(plan)) call check(sht_final(plan), 'wa_Finalize')
    plan = c_null_ptr
    if (allocated(x_Lon)) deallocate(x_Lon, y_Lat, x_Lon_Weight, y_Lat_Weight, xy_Lon, xy_Lat, rn)
  end subroutine wa_Finalize

  integer function l_nm(n, m)
    integer, intent(in) :: n, m
    l_nm = n*(n + 1) + m + 1
  end function l_nm

  function nm_l(l)
    integer, intent(in) :: l
    integer :: nm_l(2), n
    n = int(sqrt(real(l - 1, DP)))
    do while ((n + 1)**2 <= l - 1); n = n + 1; end do
    do while (n*n > l - 1); n = n - 1; end do
    nm_l(1) = n; nm_l(2) = (l - 1) - n*(n + 1)
  end function nm_l

  function w_xy(xy)
    real(DP), intent(in) :: xy(0:im-1, jm)
    real(DP) :: w_xy(lm)
    call check(sht_wa_xya(plan, xy, 1_c_int, w_xy), 'w_xy')
  end function w_xy

  function xy_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: xy_w(0:im-1, jm)
    call check(sht_xya_wa(plan, w, 1_c_int, xy_w), 'xy_w')
  end function xy_w

  function wa_xya(xya)
    real(DP), intent(in) :: xya(:,:,:)
    real(DP) :: wa_xya(lm, size(xya, 3))
    call check(sht_wa_xya(plan, xya, int(size(xya, 3), c_int), wa_xya), 'wa_xya')
  end function wa_xya

  function xya_wa(wa)
    real(DP), intent(in) :: wa(:,:)
    real(DP) :: xya_wa(0:im-1, jm, size(wa, 2))
    call check(sht_xya_wa(plan, wa, int(size(wa, 2), c_int), xya_wa), 'xya_wa')
  end function xya_wa

  function w_DivLambda_xy(xy)
    real(DP), intent(in) :: xy(0:im-1, jm)
    real(DP) :: w_DivLambda_xy(lm)
    call check(sht_wa_divlambda_xya(plan, xy, 1_c_int, w_DivLambda_xy), 'w_DivLambda_xy')
  end function w_DivLambda_xy

  function w_DivMu_xy(xy)
    real(DP), intent(in) :: xy(0:im-1, jm)
    real(DP) :: w_DivMu_xy(lm)
    call check(sht_wa_divmu_xya(plan, xy, 1_c_int, w_DivMu_xy), 'w_DivMu_xy')
  end function w_DivMu_xy

  function xy_GradLambda_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: xy_GradLambda_w(0:im-1, jm)
    call check(sht_xya_gradlambda_wa(plan, w, 1_c_int, xy_GradLambda_w), 'xy_GradLambda_w')
  end function xy_GradLambda_w

  function xy_GradMu_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: xy_GradMu_w(0:im-1, jm)
    call check(sht_xya_gradmu_wa(plan, w, 1_c_int, xy_GradMu_w), 'xy_GradMu_w')
  end function xy_GradMu_w

  function xy_GradLon_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: xy_GradLon_w(0:im-1, jm)
    call check(sht_xya_gradlon_wa(plan, w, 1_c_int, xy_GradLon_w), 'xy_GradLon_w')
  end function xy_GradLon_w

  function xy_GradLat_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: xy_GradLat_w(0:im-1, jm)
    call check(sht_xya_gradlat_wa(plan, w, 1_c_int, xy_GradLat_w), 'xy_GradLat_w')
  end function xy_GradLat_w

  function xya_GradLambda_wa(wa)
    real(DP), intent(in) :: wa(:,:)
    real(DP) :: xya_GradLambda_wa(0:im-1, jm, size(wa, 2))
    call check(sht_xya_gradlambda_wa(plan, wa, int(size(wa, 2), c_int), xya_GradLambda_wa), 'xya_GradLambda_wa')
  end function xya_GradLambda_wa

  function xya_GradMu_wa(wa)
    real(DP), intent(in) :: wa(:,:)
    real(DP) :: xya_GradMu_wa(0:im-1, jm, size(wa, 2))
    call check(sht_xya_gradmu_wa(plan, wa, int(size(wa, 2), c_int), xya_GradMu_wa), 'xya_GradMu_wa')
  end function xya_GradMu_wa

  function xya_GradLon_wa(wa)
    real(DP), intent(in) :: wa(:,:)
    real(DP) :: xya_GradLon_wa(0:im-1, jm, size(wa, 2))
    call check(sht_xya_gradlon_wa(plan, wa, int(size(wa, 2), c_int), xya_GradLon_wa), 'xya_GradLon_wa')
  end function xya_GradLon_wa

  function xya_GradLat_wa(wa)
    real(DP), intent(in) :: wa(:,:)
    real(DP) :: xya_GradLat_wa(0:im-1, jm, size(wa, 2))
    call check(sht_xya_gradlat_wa(plan, wa, int(size(wa, 2), c_int), xya_GradLat_wa), 'xya_GradLat_wa')
  end function xya_GradLat_wa

  function w_Lapla_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: w_Lapla_w(lm)
    call check(sht_wa_lapla_wa(plan, w, 1_c_int, w_Lapla_w), 'w_Lapla_w')
  end function w_Lapla_w

  function w_LaplaInv_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: w_LaplaInv_w(lm)
    call check(sht_wa_laplainv_wa(plan, w, 1_c_int, w_LaplaInv_w), 'w_LaplaInv_w')
  end function w_LaplaInv_w

  real(DP) function AvrLonLat_xy(xy)
    real(DP), intent(in) :: xy(0:im-1, jm)
    real(DP) :: r(1)
    call check(sht_avrlonlat_xya(plan, xy, 1_c_int, r), 'AvrLonLat_xy')
    AvrLonLat_xy = r(1)
  end function AvrLonLat_xy

  real(DP) function IntLonLat_xy(xy)
    real(DP), intent(in) :: xy(0:im-1, jm)
    real(DP) :: r(1)
    call check(sht_intlonlat_xya(plan, xy, 1_c_int, r), 'IntLonLat_xy')
    IntLonLat_xy = r(1)
  end function IntLonLat_xy

  function ya_AvrLon_xya(xya)
    real(DP), intent(in) :: xya(:,:,:)
    real(DP) :: ya_AvrLon_xya(jm, size(xya, 3))
    call check(sht_ya_avrlon_xya(plan, xya, int(size(xya, 3), c_int), ya_AvrLon_xya), 'ya_AvrLon_xya')
  end function ya_AvrLon_xya

  function ya_IntLon_xya(xya)
    real(DP), intent(in) :: xya(:,:,:)
    real(DP) :: ya_IntLon_xya(jm, size(xya, 3))
    call check(sht_ya_intlon_xya(plan, xya, int(size(xya, 3), c_int), ya_IntLon_xya), 'ya_IntLon_xya')
  end function ya_IntLon_xya

  ! ---- fused forms of SpmlUtil_mod's composites (one call for all levels)

  !> wa_AlphaOptr_xya (SpmlUtil_mod.f90:453-473): (DivLambda(A) + DivMu(B)) / a
  function b200_wa_AlphaOptr_xya(xya_A, xya_B)
    real(DP), intent(in) :: xya_A(:,:,:), xya_B(:,:,:)
    real(DP) :: b200_wa_AlphaOptr_xya(lm, size(xya_A, 3))
    call check(sht_wa_alphaoptr_xya(plan, xya_A, xya_B, int(size(xya_A, 3), c_int), b200_wa_AlphaOptr_xya), &
         'wa_AlphaOptr_xya')
  end function b200_wa_AlphaOptr_xya

  !> xya_AlphaOptr_wa (SpmlUtil_mod.f90:430-451): (GradLambda(A) + GradMu(B)) / (a cos^2 phi)
  function b200_xya_AlphaOptr_wa(wa_A, wa_B)
    real(DP), intent(in) :: wa_A(:,:), wa_B(:,:)
    real(DP) :: b200_xya_AlphaOptr_wa(0:im-1, jm, size(wa_A, 2))
    call check(sht_xya_alphaoptr_wa(plan, wa_A, wa_B, int(size(wa_A, 2), c_int), b200_xya_AlphaOptr_wa), &
         'xya_AlphaOptr_wa')
  end function b200_xya_AlphaOptr_wa

  !> calc_UVCosLat2VorDiv_xya_wa (SpmlUtil_mod.f90:342-368)
  subroutine b200_calc_UVCosLat2VorDiv(xya_UCosLat, xya_VCosLat, wa_Vor, wa_Div)
    real(DP), intent(in) :: xya_UCosLat(:,:,:), xya_VCosLat(:,:,:)
    real(DP), intent(out) :: wa_Vor(:,:), wa_Div(:,:)
    call check(sht_uvcoslat2vordiv(plan, xya_UCosLat, xya_VCosLat, int(size(xya_UCosLat, 3), c_int), &
         wa_Vor, wa_Div), 'calc_UVCosLat2VorDiv')
  end subroutine b200_calc_UVCosLat2VorDiv

  !> calc_VorDiv2UV_wa_xya (SpmlUtil_mod.f90:370-396)
  subroutine b200_calc_VorDiv2UV(wa_Vor, wa_Div, xya_U, xya_V)
    real(DP), intent(in) :: wa_Vor(:,:), wa_Div(:,:)
    real(DP), intent(out) :: xya_U(:,:,:), xya_V(:,:,:)
    call check(sht_vordiv2uv(plan, wa_Vor, wa_Div, int(size(wa_Vor, 2), c_int), xya_U, xya_V), 'calc_VorDiv2UV')
  end subroutine b200_calc_VorDiv2UV

  !> wa <- w_Filter * wa / (1 - dt c) (physics/DOGCM_Phys_hspm_vfvm_mod.f90:638-641, 741-742)
  subroutine b200_wa_Diffuse(wa, coef, dt, w_Filter)
    real(DP), intent(inout) :: wa(:,:)
    real(DP), intent(in) :: coef(:), dt, w_Filter(:)
    call check(sht_wa_diffuse(plan, wa, int(size(wa, 2), c_int), coef, real(dt, c_double), w_Filter), 'wa_Diffuse')
  end subroutine b200_wa_Diffuse

  !> wa_AlphaOptr_xya(A Q, B Q), products formed in the longitude transform
  !> (dynamics/hspm_vfvm/HBEBaroc_hspm_vfvm_mod.f90:160-165, Q = H cos(phi) T)
  function b200_wa_AlphaOptrProd_xya(xya_A, xya_B, xya_Q)
    real(DP), intent(in) :: xya_A(:,:,:), xya_B(:,:,:), xya_Q(:,:,:)
    real(DP) :: b200_wa_AlphaOptrProd_xya(lm, size(xya_A, 3))
    call check(sht_wa_alphaoptr_prod_xya(plan, xya_A, xya_B, xya_Q, int(size(xya_A, 3), c_int), &
         b200_wa_AlphaOptrProd_xya), 'wa_AlphaOptrProd_xya')
  end function b200_wa_AlphaOptrProd_xya

  !> calc_UVCosLat2VorDiv(cos(phi) (X1 Q + Z1), cos(phi) (X2 Q + Z2)): xy_A, xy_B of
  !> HBEBaroc_MOMRHS_VorDivForm (dynamics/hspm_vfvm/HBEBaroc_hspm_vfvm_mod.f90:394-418)
  !> formed in the longitude transform (Q = Vor, X1 = U, X2 = V, Z1, Z2 the other terms)
  subroutine b200_calc_MomProd2VorDiv(xya_X1, xya_X2, xya_Q, xya_Z1, xya_Z2, wa_Vor, wa_Div)
    real(DP), intent(in) :: xya_X1(:,:,:), xya_X2(:,:,:), xya_Q(:,:,:), xya_Z1(:,:,:), xya_Z2(:,:,:)
    real(DP), intent(out) :: wa_Vor(:,:), wa_Div(:,:)
    call check(sht_uvcoslat2vordiv_fma(plan, xya_X1, xya_X2, xya_Q, xya_Z1, xya_Z2, &
         int(size(xya_X1, 3), c_int), wa_Vor, wa_Div), 'calc_MomProd2VorDiv')
  end subroutine b200_calc_MomProd2VorDiv

  !> xya_GradLon_wa and xya_GradLat_wa of one spectrum, one synthesis
  subroutine b200_xya_HGrad_wa(wa, xya_GradLon, xya_GradLat)
    real(DP), intent(in) :: wa(:,:)
    real(DP), intent(out) :: xya_GradLon(:,:,:), xya_GradLat(:,:,:)
    call check(sht_xya_hgrad_wa(plan, wa, int(size(wa, 2), c_int), xya_GradLon, xya_GradLat), 'xya_HGrad_wa')
  end subroutine b200_xya_HGrad_wa

  !> xya_GradLon_wa(wa_xya(T)), xya_GradLat_wa(wa_xya(T)): the Redi/GM tracer
  !> gradients before 1/RPlanet (physics/lphys/LPhys_RediGM_hspm_vfvm_mod.f90:432-440)
  subroutine b200_xya_HGrad_xya(xya, xya_GradLon, xya_GradLat)
    real(DP), intent(in) :: xya(:,:,:)
    real(DP), intent(out) :: xya_GradLon(:,:,:), xya_GradLat(:,:,:)
    call check(sht_xya_hgrad_xya(plan, xya, int(size(xya, 3), c_int), xya_GradLon, xya_GradLat), 'xya_HGrad_xya')
  end subroutine b200_xya_HGrad_xya

  !> xya_wa(wa_AlphaOptr_xya(A, B)) grid to grid: the Redi/GM flux divergence
  !> (physics/lphys/LPhys_RediGM_hspm_vfvm_mod.f90:350-355)
  function b200_xya_FluxDiv_xya(xya_A, xya_B)
    real(DP), intent(in) :: xya_A(:,:,:), xya_B(:,:,:)
    real(DP) :: b200_xya_FluxDiv_xya(0:im-1, jm, size(xya_A, 3))
    call check(sht_xya_fluxdiv_xya(plan, xya_A, xya_B, int(size(xya_A, 3), c_int), b200_xya_FluxDiv_xya), &
         'xya_FluxDiv_xya')
  end function b200_xya_FluxDiv_xya

  !> wa_xya of the section xyz(is:is+im-1, js:js+jm-1, :) of a haloed array
  !> xyz(IA, JA, KA) (util/grid/DOGCM_GaussSpmVFvmGrid_mod.f90:158-183; with
  !> the model's one-point halos is = js = 2), read in place through the
  !> array's leading dimensions instead of an explicit-shape section copy.
  !> mode: SHT_PREC_FP64 / SHT_PREC_SPLIT for this call (default: the plan's).
  function b200_wa_xyz_section(xyz, is, js, mode)
    real(DP), intent(in), contiguous, target :: xyz(:,:,:)
    integer, intent(in) :: is, js
    integer, intent(in), optional :: mode
    real(DP) :: b200_wa_xyz_section(lm, size(xyz, 3))
    integer(c_int) :: md
    md = -1
    if (present(mode)) md = int(mode, c_int)
    if (is < 1 .or. js < 1 .or. is + im - 1 > size(xyz, 1) .or. js + jm - 1 > size(xyz, 2)) &
         call MessageNotify('E', module_name, 'wa_xyz_section: section outside the array')
    call check(sht_analysis(plan, c_loc(xyz(is, js, 1)), int(size(xyz, 1), c_int), int(size(xyz, 2), c_int), &
         int(size(xyz, 3), c_int), b200_wa_xyz_section, int(lm, c_int), md), 'wa_xyz_section')
  end function b200_wa_xyz_section

  !> xya_wa into the section xyz(is:is+im-1, js:js+jm-1, :) of a haloed array;
  !> the halo points keep their values.  wa(LW, KA) with LW >= lm.
  subroutine b200_xyz_wa_section(wa, xyz, is, js, mode)
    real(DP), intent(in) :: wa(:,:)
    real(DP), intent(inout), contiguous, target :: xyz(:,:,:)
    integer, intent(in) :: is, js
    integer, intent(in), optional :: mode
    integer(c_int) :: md
    md = -1
    if (present(mode)) md = int(mode, c_int)
    if (is < 1 .or. js < 1 .or. is + im - 1 > size(xyz, 1) .or. js + jm - 1 > size(xyz, 2) .or. &
         size(wa, 2) /= size(xyz, 3)) &
         call MessageNotify('E', module_name, 'xyz_wa_section: section outside the array')
    call check(sht_synthesis(plan, wa, int(size(wa, 1), c_int), int(size(wa, 2), c_int), c_loc(xyz(is, js, 1)), &
         int(size(xyz, 1), c_int), int(size(xyz, 2), c_int), md), 'xyz_wa_section')
  end subroutine b200_xyz_wa_section

  ! ------------------------------------------------------------------------
  ! Legacy spellings (sogcm SpmlUtil_mod): the same batched transforms with the
  ! vertical index 0:km last (wz, xyz) or 0:tm (wt, xyt on Chebyshev points).

  !> xyz_wz = xya_wa (model/old/sogcm/util/SpmlUtil_mod.f90:308-320)
  function xyz_wz(wz)
    real(DP), intent(in) :: wz(:,0:)
    real(DP) :: xyz_wz(0:im-1, jm, 0:size(wz, 2) - 1)
    call check(sht_xya_wa(plan, wz, int(size(wz, 2), c_int), xyz_wz), 'xyz_wz')
  end function xyz_wz

  !> wz_xyz = wa_xya (model/old/sogcm/util/SpmlUtil_mod.f90:322-333)
  function wz_xyz(xyz)
    real(DP), intent(in) :: xyz(:,:,0:)
    real(DP) :: wz_xyz(lm, 0:size(xyz, 3) - 1)
    call check(sht_wa_xya(plan, xyz, int(size(xyz, 3), c_int), wz_xyz), 'wz_xyz')
  end function wz_xyz

  !> wt_xyt = wa_xya on the Chebyshev levels (model/old/sogcm/util/SpmlUtil_mod.f90:335-346)
  function wt_xyt(xyt)
    real(DP), intent(in) :: xyt(:,:,0:)
    real(DP) :: wt_xyt(lm, 0:size(xyt, 3) - 1)
    call check(sht_wa_xya(plan, xyt, int(size(xyt, 3), c_int), wt_xyt), 'wt_xyt')
  end function wt_xyt

  !> (wa_DivLambda_xya(A) + wa_DivMu_xya(B)) / Radius (model/old/sogcm/util/SpmlUtil_mod.f90:529-543)
  function wz_AlphaOptr_xyz(xyz_A, xyz_B)
    real(DP), intent(in) :: xyz_A(:,:,0:), xyz_B(:,:,0:)
    real(DP) :: wz_AlphaOptr_xyz(lm, 0:size(xyz_A, 3) - 1)
    call check(sht_wa_alphaoptr_xya(plan, xyz_A, xyz_B, int(size(xyz_A, 3), c_int), wz_AlphaOptr_xyz), &
         'wz_AlphaOptr_xyz')
  end function wz_AlphaOptr_xyz

  !> (xya_GradLambda_wa(A) + xya_GradMu_wa(B)) / (Radius cos^2 phi)
  !> (model/old/sogcm/util/SpmlUtil_mod.f90:561-577)
  function xyz_AlphaOptr_wz(wz_A, wz_B)
    real(DP), intent(in) :: wz_A(:,0:), wz_B(:,0:)
    real(DP) :: xyz_AlphaOptr_wz(0:im-1, jm, 0:size(wz_A, 2) - 1)
    call check(sht_xya_alphaoptr_wa(plan, wz_A, wz_B, int(size(wz_A, 2), c_int), xyz_AlphaOptr_wz), &
         'xyz_AlphaOptr_wz')
  end function xyz_AlphaOptr_wz

  !> w_Lapla_w / Radius**2 (model/old/sogcm/util/SpmlUtil_mod.f90:596-615)
  function w_Lapla2D_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: w_Lapla2D_w(lm)
    call check(sht_wa_lapla_wa(plan, w, 1_c_int, w_Lapla2D_w), 'w_Lapla2D_w')
    w_Lapla2D_w = w_Lapla2D_w / radius_**2
  end function w_Lapla2D_w

  !> wa_Lapla_wa / Radius**2 (model/old/sogcm/util/SpmlUtil_mod.f90:617-636)
  function wz_Lapla2D_wz(wz)
    real(DP), intent(in) :: wz(:,0:)
    real(DP) :: wz_Lapla2D_wz(lm, 0:size(wz, 2) - 1)
    call check(sht_wa_lapla_wa(plan, wz, int(size(wz, 2), c_int), wz_Lapla2D_wz), 'wz_Lapla2D_wz')
    wz_Lapla2D_wz = wz_Lapla2D_wz / radius_**2
  end function wz_Lapla2D_wz

  !> w_LaplaInv_w * Radius**2 (model/old/sogcm/util/SpmlUtil_mod.f90:660-679)
  function w_InvLapla2D_w(w)
    real(DP), intent(in) :: w(lm)
    real(DP) :: w_InvLapla2D_w(lm)
    call check(sht_wa_laplainv_wa(plan, w, 1_c_int, w_InvLapla2D_w), 'w_InvLapla2D_w')
    w_InvLapla2D_w = w_InvLapla2D_w * radius_**2
  end function w_InvLapla2D_w

  !> wa_LaplaInv_wa * Radius**2 (model/old/sogcm/util/SpmlUtil_mod.f90:638-657)
  function wz_InvLapla2D_wz(wz)
    real(DP), intent(in) :: wz(:,0:)
    real(DP) :: wz_InvLapla2D_wz(lm, 0:size(wz, 2) - 1)
    call check(sht_wa_laplainv_wa(plan, wz, int(size(wz, 2), c_int), wz_InvLapla2D_wz), 'wz_InvLapla2D_wz')
    wz_InvLapla2D_wz = wz_InvLapla2D_wz * radius_**2
  end function wz_InvLapla2D_wz

end module wa_module_b200
