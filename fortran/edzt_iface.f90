! edzt_iface.f90 -- iso_c_binding interfaces of libedzt (include/edzt.h) for
! the reference's Fortran host (yw-choi/DMFT-ED-ZT).
!
! Add this file to the reference's src/Makefile OBJS ahead of the modules
! that use it, and link with -L<dir> -ledzt -lcudart.  Every function returns
! an EDZT_* status; edzt_check turns a non-zero status into the reference's
! abort, die() of the fdf utils module (src/fdf/utils.F90).
!
! Seeds: the C ABI takes uint64_t seeds.  Fortran has no unsigned integers,
! so they are bound as integer(c_int64_t), value, which has the same size
! and passing convention: the library receives the same 64 bits.  A seed s
! >= 2**63 is passed as s - 2**64 (its two's-complement bit pattern), e.g.
! with transfer() from an integer(c_int8_t) array or by writing the negative
! literal; seeds below 2**63 are passed as they are.
module edzt_iface
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: EDZT_OK = 0
  interface
    integer(c_int) function edzt_ctx_create(device, ctx) bind(C, name="edzt_ctx_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr) :: ctx
    end function
    subroutine edzt_ctx_destroy(ctx) bind(C, name="edzt_ctx_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine
    type(c_ptr) function edzt_last_error(ctx) bind(C, name="edzt_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edzt_set_model(ctx, norb, nbath, em, ek, vmk, U, Up, Jex, Jp, mu) &
        bind(C, name="edzt_set_model")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: norb, nbath
      real(c_double), intent(in) :: em(*), ek(*), vmk(*)      ! em(norb,2), ek(nbath,2), vmk(norb,nbath,2)
      real(c_double), value :: U, Up, Jex, Jp, mu
    end function
    integer(c_int) function edzt_hx(ctx, ne_up, ne_dn, x, y, accumulate) bind(C, name="edzt_hx")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ne_up, ne_dn, accumulate
      real(c_double), intent(in) :: x(*)
      real(c_double), intent(inout) :: y(*)
    end function
    integer(c_int) function edzt_apply_c(ctx, ne_up, ne_dn, vec, pm, iorb, ispin, vec_out) &
        bind(C, name="edzt_apply_c")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ne_up, ne_dn, pm, iorb, ispin
      real(c_double), intent(in) :: vec(*)
      real(c_double), intent(out) :: vec_out(*)
    end function
    integer(c_int) function edzt_lanczos_iteration(ctx, ne_up, ne_dn, v_init, maxnstep, nstep, a, b) &
        bind(C, name="edzt_lanczos_iteration")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ne_up, ne_dn, maxnstep
      real(c_double), intent(in) :: v_init(*)
      integer(c_int), intent(out) :: nstep
      real(c_double), intent(out) :: a(*), b(*)
    end function
    integer(c_int) function edzt_diag_lanczos(ctx, ne_up, ne_dn, maxnstep, seed, stream, eigval, eigvec, &
        residual) bind(C, name="edzt_diag_lanczos")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: ne_up, ne_dn, maxnstep
      integer(c_int64_t), value :: seed, stream
      real(c_double), intent(out) :: eigval, eigvec(*), residual
    end function
    integer(c_int) function edzt_diag_arpack(ctx, ne_up, ne_dn, seed, stream, eigval, eigvec, ritz, resid, &
        nmult) bind(C, name="edzt_diag_arpack")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: ne_up, ne_dn
      integer(c_int64_t), value :: seed, stream
      real(c_double), intent(out) :: eigval, eigvec(*), ritz(3), resid(3)
      integer(c_int), intent(out) :: nmult
    end function
    integer(c_int) function edzt_set_diag_solver(ctx, diag_solver) bind(C, name="edzt_set_diag_solver")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: diag_solver                    ! 1 Lanczos, 2 ARPACK
    end function
    integer(c_int) function edzt_set_keep_vectors(ctx, keep) bind(C, name="edzt_set_keep_vectors")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: keep                           ! 1 keep when they fit, 0 rerun
    end function
    integer(c_int) function edzt_ground_state(ctx, nsector, sectors, maxnstep, seed, isector, e0, gsvec, &
        e_sector) bind(C, name="edzt_ground_state")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsector, maxnstep
      integer(c_int), intent(in) :: sectors(*)                 ! (2, nsector): ne_up, ne_dn
      integer(c_int64_t), value :: seed
      integer(c_int), intent(out) :: isector                   ! 0-based
      real(c_double), intent(out) :: e0, gsvec(*), e_sector(*)
    end function
    integer(c_long_long) function edzt_gs_dim(ctx) bind(C, name="edzt_gs_dim")
      import :: c_long_long, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edzt_green_diag(ctx, iorb, ispin, maxnstep, nw, omega, ap, bp, am, bm, g) &
        bind(C, name="edzt_green_diag")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: ctx
      integer(c_int), value :: iorb, ispin, maxnstep, nw
      real(c_double), intent(in) :: omega(*)
      real(c_double), intent(out) :: ap(*), bp(*), am(*), bm(*)
      complex(c_double_complex), intent(out) :: g(*)
    end function
    integer(c_int) function edzt_cluster_green_ftn(ctx, nspin, maxnstep, nw, omega, G_cl, coeffs) &
        bind(C, name="edzt_cluster_green_ftn")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: ctx
      integer(c_int), value :: nspin, maxnstep, nw
      real(c_double), intent(in) :: omega(*)
      complex(c_double_complex), intent(out) :: G_cl(*)         ! G_cl(nw, norb, nspin)
      real(c_double), intent(out) :: coeffs(*)                  ! (maxnstep, 4, 2, norb)
    end function
    integer(c_int) function edzt_solve(ctx, nsector, sectors, maxnstep, seed, nspin, nw, omega, isector, e0, &
        G_cl, coeffs) bind(C, name="edzt_solve")
      import :: c_int, c_ptr, c_double, c_double_complex, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsector, maxnstep, nspin, nw
      integer(c_int), intent(in) :: sectors(*)                 ! (2, nsector)
      integer(c_int64_t), value :: seed
      real(c_double), intent(in) :: omega(*)
      integer(c_int), intent(out) :: isector                   ! 0-based
      real(c_double), intent(out) :: e0
      complex(c_double_complex), intent(out) :: G_cl(*)       ! G_cl(nw, norb, nspin)
      real(c_double), intent(out) :: coeffs(*)                 ! (maxnstep, 4, 2, norb)
    end function
    ! post_process (src/post_process.f90) on the resident ground state
    integer(c_int) function edzt_gs_occupancy(ctx, nspin, occ, docc) bind(C, name="edzt_gs_occupancy")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nspin
      real(c_double), intent(out) :: occ(*), docc(*)           ! occ(norb, nspin), docc(norb)
    end function
    integer(c_int) function edzt_green_real(ctx, iorb, ispin, maxnstep, nw, omega, eta, g) &
        bind(C, name="edzt_green_real")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: ctx
      integer(c_int), value :: iorb, ispin, maxnstep, nw
      real(c_double), intent(in) :: omega(*)                   ! real frequencies
      real(c_double), value :: eta
      complex(c_double_complex), intent(out) :: g(*)          ! A(w) = -aimag(g) / pi
    end function
    integer(c_int) function edzt_cluster_green_matrix(ctx, nspin, maxnstep, nw, omega, G) &
        bind(C, name="edzt_cluster_green_matrix")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: ctx
      integer(c_int), value :: nspin, maxnstep, nw
      real(c_double), intent(in) :: omega(*)
      complex(c_double_complex), intent(out) :: G(*)          ! G_ab(nw, norb, norb, nspin)
    end function
    ! the C library's strlen, for the error message
    integer(c_size_t) function edzt_c_strlen(s) bind(C, name="strlen")
      import :: c_size_t, c_ptr
      type(c_ptr), value :: s
    end function
  end interface
contains
  ! Abort through the reference's die() when rc is not EDZT_OK, with the
  ! context's error message (edzt_last_error).
  subroutine edzt_check(ctx, rc)
    use utils, only: die
    type(c_ptr), intent(in) :: ctx
    integer(c_int), intent(in) :: rc
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    character(len=:), allocatable :: msg
    integer :: i, n
    if (rc == EDZT_OK) return
    p = edzt_last_error(ctx)
    n = int(edzt_c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate(character(len=n) :: msg)
    do i = 1, n
      msg(i:i) = chars(i)
    end do
    call die("edzt", msg)
  end subroutine
end module edzt_iface
