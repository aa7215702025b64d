!===============================================================================
! rgf_iface.f90 -- ISO_C_BINDING interface to librgf_b200.so (include/rgf.h).
!
! Drop-in for the liteQT RGF routines:
!   green_RGF_RS  (src/green_rgf.f90:3950, module green_rgf)
!   RGF_G         (src/rgf_mod.f90:26,     module rgf_mod)
!   green_RGF_CMS (src/green_rgf.f90:4167, module green_rgf; overlap Sii)
! The wrappers below keep the reference's argument lists, so the call sites
! (green_rgf.f90:2918-2923, :3174-3178, :735-739, :970-974, gw_sparse.f90:285-292)
! compile unchanged once `use rgf_cuda` replaces the module-local routine.
! The batched entry point rgf_solve_energies replaces a whole `!$omp do ie`
! loop with one launch.
!
! Integer kinds: dimensions cross the ABI as integer(c_int64_t), so the module
! works both with default 4-byte integers and with -i8 (Makefile.intel:6).
!===============================================================================
module rgf_cuda
  use, intrinsic :: iso_c_binding
  implicit none
  private
  public :: green_RGF_RS, RGF_G, green_RGF_CMS, rgf_solve_energies_f, rgf_device_t, rgf_task_info_t

  type, bind(C) :: rgf_device_t
    integer(c_int64_t) :: nm, nx
    type(c_ptr) :: Hii, H1i
    real(c_double) :: mu(2), temp(2)
    type(c_ptr) :: Sii
  end type rgf_device_t

  type, bind(C) :: rgf_task_info_t
    integer(c_int32_t) :: status, sancho_iters_left, sancho_iters_right, n_gemm, n_inv, reserved
  end type rgf_task_info_t

  interface
    integer(c_int) function c_rgf_green_rgf_rs(ctx, temp, nm, nx, E, mu, Hii, H1i, sl, sg, sr, &
        ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1) bind(C, name="rgf_green_rgf_rs")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: temp(2), E, mu(2)
      integer(c_int64_t), intent(in) :: nm, nx
      type(c_ptr), value :: Hii, H1i, sl, sg, sr, ndens, pdens, ldos, cur, GRi1, GLi1, GGi1
      real(c_double), intent(inout) :: tr, tre
    end function c_rgf_green_rgf_rs

    integer(c_int) function c_rgf_rgf_g(ctx, temp, nm, nx, E, mu, Hii, H1i, sl, sg, sr, &
        tr, tre, ndens, pdens, ldos, cur, GRi1, GLi1, GGi1) bind(C, name="rgf_rgf_g")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: temp(2), E, mu(2)
      integer(c_int64_t), intent(in) :: nm, nx
      type(c_ptr), value :: Hii, H1i, sl, sg, sr, ndens, pdens, ldos, cur, GRi1, GLi1, GGi1
      real(c_double), intent(inout) :: tr, tre
    end function c_rgf_rgf_g

    integer(c_int) function c_rgf_green_rgf_cms(ctx, temp, nm, nx, E, mu, Sii, Hii, H1i, sl, sg, sr, &
        ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1) bind(C, name="rgf_green_rgf_cms")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: temp(2), E, mu(2)
      integer(c_int64_t), intent(in) :: nm, nx
      type(c_ptr), value :: Sii, Hii, H1i, sl, sg, sr, ndens, pdens, ldos, cur, GRi1, GLi1, GGi1
      real(c_double), intent(inout) :: tr, tre
    end function c_rgf_green_rgf_cms

    integer(c_int) function c_rgf_solve_energies(ctx, device, nen, E, sl, sr, ldos, ndens, pdens, &
        GRi1, cur, tr, tre, T, info, stream) bind(C, name="rgf_solve_energies")
      import :: c_int, c_ptr, c_int64_t, rgf_device_t
      type(c_ptr), value :: ctx
      type(rgf_device_t), intent(in) :: device
      integer(c_int64_t), value :: nen
      type(c_ptr), value :: E, sl, sr, ldos, ndens, pdens, GRi1, cur, tr, tre, T, info, stream
    end function c_rgf_solve_energies

    integer(c_int) function c_rgf_ctx_create(opts, ctx) bind(C, name="rgf_ctx_create")
      import :: c_int, c_ptr
      type(c_ptr), value :: opts
      type(c_ptr), intent(out) :: ctx
    end function c_rgf_ctx_create

    type(c_ptr) function c_rgf_last_error() bind(C, name="rgf_last_error")
      import :: c_ptr
    end function c_rgf_last_error
  end interface

contains

  ! NULL for an absent optional argument, else its address.
  function opt_ptr(a) result(p)
    complex(8), intent(inout), target, optional :: a(:,:,:)
    type(c_ptr) :: p
    if (present(a)) then
      p = c_loc(a)
    else
      p = c_null_ptr
    end if
  end function opt_ptr

  subroutine check(rc, who)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: who
    if (rc /= 0) then
      print *, 'SEVERE warning: ', who, ' failed, rc=', rc
    end if
  end subroutine check

  ! green_RGF_RS with the reference's argument list (src/green_rgf.f90:3950).
  subroutine green_RGF_RS(TEMP, nm, nx, E, mu, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, &
      sigma_r_ph, ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1)
    integer, intent(in) :: nm, nx
    real(8), intent(in) :: E, mu(2), temp(2)
    complex(8), intent(in), target, dimension(nm,nm,nx) :: sigma_lesser_ph, sigma_greater_ph, sigma_r_ph
    complex(8), intent(in), target, dimension(nm,nm,nx) :: Hii, H1i
    complex(8), intent(inout), target, dimension(nm,nm,nx) :: ldos, ndens, pdens
    real(8), intent(inout), target, dimension(nm,nm,nx) :: cur
    complex(8), intent(inout), target, dimension(nm,nm,nx), optional :: GRi1, GLi1, GGi1
    real(8), intent(inout) :: tr, tre
    integer(c_int64_t) :: nm8, nx8
    integer(c_int) :: rc
    nm8 = nm
    nx8 = nx
    rc = c_rgf_green_rgf_rs(c_null_ptr, temp, nm8, nx8, E, mu, c_loc(Hii), c_loc(H1i), &
        c_loc(sigma_lesser_ph), c_loc(sigma_greater_ph), c_loc(sigma_r_ph), c_loc(ndens), &
        c_loc(pdens), c_loc(ldos), tr, tre, c_loc(cur), opt_ptr(GRi1), opt_ptr(GLi1), opt_ptr(GGi1))
    call check(rc, 'green_RGF_RS')
  end subroutine green_RGF_RS

  ! RGF_G with the reference's argument list (src/rgf_mod.f90:26).
  subroutine RGF_G(temperature, nm, nx, E, mu, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, &
      sigma_r_ph, tr, tre, ndens, pdens, ldos, cur, GRi1, GLi1, GGi1)
    integer, intent(in) :: nm, nx
    real(8), intent(in) :: E, mu(2), temperature(2)
    complex(8), intent(in), target, dimension(nm,nm,nx) :: sigma_lesser_ph, sigma_greater_ph, sigma_r_ph
    complex(8), intent(in), target, dimension(nm,nm,nx) :: Hii, H1i
    real(8), intent(inout) :: tr, tre
    complex(8), intent(inout), target, dimension(nm,nm,nx) :: ldos, ndens, pdens
    real(8), intent(inout), target, dimension(nm,nm,nx) :: cur
    complex(8), intent(inout), target, dimension(nm,nm,nx), optional :: GRi1, GLi1, GGi1
    integer(c_int64_t) :: nm8, nx8
    integer(c_int) :: rc
    nm8 = nm
    nx8 = nx
    rc = c_rgf_rgf_g(c_null_ptr, temperature, nm8, nx8, E, mu, c_loc(Hii), c_loc(H1i), &
        c_loc(sigma_lesser_ph), c_loc(sigma_greater_ph), c_loc(sigma_r_ph), tr, tre, &
        c_loc(ndens), c_loc(pdens), c_loc(ldos), c_loc(cur), opt_ptr(GRi1), opt_ptr(GLi1), opt_ptr(GGi1))
    call check(rc, 'RGF_G')
  end subroutine RGF_G

  ! green_RGF_CMS with the reference's argument list (src/green_rgf.f90:4167).
  subroutine green_RGF_CMS(TEMP, nm, nx, E, mu, Sii, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, &
      sigma_r_ph, ndens, pdens, ldos, tr, tre, cur, GRi1, GLi1, GGi1)
    integer, intent(in) :: nm, nx
    real(8), intent(in) :: E, mu(2), temp(2)
    complex(8), intent(in), target, dimension(nm,nm,nx) :: sigma_lesser_ph, sigma_greater_ph, sigma_r_ph
    complex(8), intent(in), target, dimension(nm,nm,nx) :: Sii, Hii, H1i
    complex(8), intent(inout), target, dimension(nm,nm,nx) :: ldos, ndens, pdens
    real(8), intent(inout), target, dimension(nm,nm,nx) :: cur
    complex(8), intent(inout), target, dimension(nm,nm,nx), optional :: GRi1, GLi1, GGi1
    real(8), intent(inout) :: tr, tre
    integer(c_int64_t) :: nm8, nx8
    integer(c_int) :: rc
    nm8 = nm
    nx8 = nx
    rc = c_rgf_green_rgf_cms(c_null_ptr, temp, nm8, nx8, E, mu, c_loc(Sii), c_loc(Hii), c_loc(H1i), &
        c_loc(sigma_lesser_ph), c_loc(sigma_greater_ph), c_loc(sigma_r_ph), c_loc(ndens), &
        c_loc(pdens), c_loc(ldos), tr, tre, c_loc(cur), opt_ptr(GRi1), opt_ptr(GLi1), opt_ptr(GGi1))
    call check(rc, 'green_RGF_CMS')
  end subroutine green_RGF_CMS

  ! All energies of one k-point in one launch: replaces
  !   !$omp do; do ie=1,nen; call green_RGF_RS(...); enddo
  ! (green_rgf.f90:2916-2925) for arrays g(nm,nm,nx,nen).
  subroutine rgf_solve_energies_f(ctx, nm, nx, nen, En, mu, temp, Hii, H1i, sigma_lesser, &
      sigma_r, g_lesser, g_greater, g_r, tr, tre, cur, g_r_i1)
    type(c_ptr), intent(in) :: ctx
    integer, intent(in) :: nm, nx, nen
    real(8), intent(in), target :: En(nen), mu(2), temp(2)
    complex(8), intent(in), target :: Hii(nm,nm,nx), H1i(nm,nm,nx)
    complex(8), intent(in), target :: sigma_lesser(nm,nm,nx,nen), sigma_r(nm,nm,nx,nen)
    complex(8), intent(inout), target :: g_lesser(nm,nm,nx,nen), g_greater(nm,nm,nx,nen)
    complex(8), intent(inout), target :: g_r(nm,nm,nx,nen), g_r_i1(nm,nm,nx,nen)
    real(8), intent(inout), target :: tr(nen), tre(nen), cur(nm,nm,nx,nen)
    type(rgf_device_t) :: dev
    integer(c_int) :: rc
    dev%nm = nm
    dev%nx = nx
    dev%Hii = c_loc(Hii)
    dev%H1i = c_loc(H1i)
    dev%mu = mu
    dev%temp = temp
    dev%Sii = c_null_ptr
    rc = c_rgf_solve_energies(ctx, dev, int(nen, c_int64_t), c_loc(En), c_loc(sigma_lesser), &
        c_loc(sigma_r), c_loc(g_r), c_loc(g_lesser), c_loc(g_greater), c_loc(g_r_i1), c_loc(cur), &
        c_loc(tr), c_loc(tre), c_null_ptr, c_null_ptr, c_null_ptr)
    call check(rc, 'rgf_solve_energies')
  end subroutine rgf_solve_energies_f

end module rgf_cuda
