! thp_shim.f90 -- ISO_C_BINDING layer between Tinker-HP (v1.2 module state)
! and libthp.so.  Replaces the calls newinduce_pme2 (epolar.f:108,
! epolar1.f:145), mlistcell (nblist.f:109), epolar1 (gradient.f:165) and
! empole1 and ehal1 (gradient.f, the permanent-multipole and vdW terms) by
! thp_newinduce_pme2, thp_mlistcell, thp_epolar1, thp_empole1 and thp_ehal1,
! and offers the batched per-site PME routines.
!
! Binding rules this file follows:
!   * It binds to the library's thp_f_* entry points, never to the
!     reference-named drop-ins (newinduce_pme2_, mlistcell_, ...): those
!     symbols are also defined by the reference's own objects, so a build
!     that keeps the reference sources links either a duplicate or the CPU
!     routine.
!   * Module arrays go to the C side as assumed-size dummy arguments (the
!     caller passes their address), not through c_loc, which requires the
!     TARGET or POINTER attribute that Tinker-HP's module variables do not
!     carry.  The library keeps the addresses given to c_bind_state,
!     c_bind_gradient, c_bind_mpole and c_bind_vdw until the next bind: pass
!     only contiguous allocatable module arrays there (x, y, z, rpole, uind,
!     uinp, nelst, elst, dep, dem, dev), for which the compiler passes the
!     array itself and no temporary copy.
!   * maxelst is a parameter of module sizes (MOD_sizes.f:58) and lbuffer a
!     variable of module neigh (MOD_neigh.f:58).
! Not compiled in this repository's image (no Fortran compiler); it follows
! the C declarations of include/thp.h.
module thp_shim
  use iso_c_binding
  implicit none
  private
  public :: thp_init, thp_newinduce_pme2, thp_mlistcell, thp_epolar, thp_epolar1, thp_empole1, thp_ehal1, &
            thp_finalize
  public :: thp_grid_uind_sites, thp_fphi_uind_sites

  type, bind(C) :: thp_config
    integer(c_int) :: n
    real(c_double) :: box(3)
    real(c_double) :: aewald, ewaldcut, lbuffer
    integer(c_int) :: nfft(3)
    integer(c_int) :: bsorder, politer
    real(c_double) :: poleps
    integer(c_int) :: precision, max_neighbors, device
  end type

  type(c_ptr), save :: ctx = c_null_ptr
  integer(c_int), allocatable, target, save :: off(:,:), idx(:,:)

  interface
    integer(c_int) function c_ctx_create(cfg, out) bind(C, name="thp_ctx_create")
      import :: c_int, c_ptr, thp_config
      type(thp_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: out
    end function
    integer(c_int) function c_ctx_destroy(h) bind(C, name="thp_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function c_set_params(h, pol, thl, pdm) bind(C, name="thp_set_params")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: pol(*), thl(*), pdm(*)
    end function
    integer(c_int) function c_set_connectivity(h, offp, idxp, scales) bind(C, name="thp_set_connectivity")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, offp, idxp, scales
    end function
    integer(c_int) function c_bind_state(h, x, y, z, rpole, uind, uinp, nelst, elst, maxelst, ep) &
        bind(C, name="thp_bind_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double) :: x(*), y(*), z(*), rpole(*), uind(*), uinp(*), ep
      integer(c_int) :: nelst(*), elst(*)
      integer(c_int), value :: maxelst
    end function
    subroutine c_newinduce_pme2() bind(C, name="thp_f_newinduce_pme2")
    end subroutine
    subroutine c_mlistcell() bind(C, name="thp_f_mlistcell")
    end subroutine
    subroutine c_epolar() bind(C, name="thp_f_epolar")
    end subroutine
    subroutine c_epolar1() bind(C, name="thp_f_epolar1")
    end subroutine
    integer(c_int) function c_set_frames(h, pole, zax, xax, axt) bind(C, name="thp_set_frames")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, pole, zax, xax, axt
    end function
    integer(c_int) function c_bind_gradient(h, dep) bind(C, name="thp_bind_gradient")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double) :: dep(*)
    end function
    integer(c_int) function c_set_mpole_scales(h, m) bind(C, name="thp_set_mpole_scales")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, m
    end function
    integer(c_int) function c_bind_mpole(h, em, dem) bind(C, name="thp_bind_mpole")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double) :: em, dem(*)
    end function
    subroutine c_empole1() bind(C, name="thp_f_empole1")
    end subroutine
    integer(c_int) function c_set_vdw(h, cls, nclass, tables, ired, kred, vscale, vdwcut, vdwtaper, &
        ghal, dhal) bind(C, name="thp_set_vdw")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h, cls, tables, ired, kred, vscale
      integer(c_int), value :: nclass
      real(c_double), value :: vdwcut, vdwtaper, ghal, dhal
    end function
    integer(c_int) function c_bind_vdw(h, ev, dev) bind(C, name="thp_bind_vdw")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double) :: ev, dev(*)
    end function
    subroutine c_ehal1() bind(C, name="thp_f_ehal1")
    end subroutine
    subroutine c_grid_uind_sites(ns, isite, fuind, fuinp, qgrid) bind(C, name="thp_f_grid_uind_sites")
      import :: c_int, c_double
      integer(c_int), intent(in) :: ns, isite(*)
      real(c_double), intent(in) :: fuind(3,*), fuinp(3,*)
      real(c_double), intent(inout) :: qgrid(*)
    end subroutine
    subroutine c_fphi_uind_sites(ns, isite, qgrid, phi1, phi2, sphi) bind(C, name="thp_f_fphi_uind_sites")
      import :: c_int, c_double
      integer(c_int), intent(in) :: ns, isite(*)
      real(c_double), intent(in) :: qgrid(*)
      real(c_double), intent(out) :: phi1(10,*), phi2(10,*), sphi(20,*)
    end subroutine
    integer(c_int) function c_last_error() bind(C, name="thp_last_error")
      import :: c_int
    end function
  end interface

contains

  ! called once from mechanic after kpolar/kmpole/kewald/cutoffs
  subroutine thp_init(mixed)
    use atoms, only: n
    use boxes, only: xbox, ybox, zbox
    use ewald, only: aewald
    use cutoff, only: ewaldcut
    use neigh, only: lbuffer
    use pme, only: nfft1, nfft2, nfft3, bsorder
    use polar, only: polarity, thole, pdamp
    use polpot, only: politer, poleps, p2scale, p3scale, p4scale, p5scale, p2iscale, p3iscale, &
                      p4iscale, p5iscale, d1scale, d2scale, d3scale, d4scale, u1scale, u2scale, &
                      u3scale, u4scale
    use mplpot, only: m2scale, m3scale, m4scale, m5scale
    use potent, only: use_vdw
    logical, intent(in) :: mixed
    type(thp_config), target :: cfg
    real(c_double), target :: scales(16), mscales(4)
    type(c_ptr), target :: offp(8), idxp(8)
    integer :: st
    cfg%n = n
    cfg%box = [xbox, ybox, zbox]
    cfg%aewald = aewald
    cfg%ewaldcut = ewaldcut
    cfg%lbuffer = lbuffer
    cfg%nfft = [nfft1, nfft2, nfft3]
    cfg%bsorder = bsorder
    cfg%politer = politer
    cfg%poleps = poleps
    cfg%precision = merge(1, 0, mixed)
    cfg%max_neighbors = 0
    cfg%device = 0
    st = c_ctx_create(cfg, ctx)
    if (st /= 0) call fatal
    st = c_set_params(ctx, polarity, thole, pdamp)  ! copied before the call returns
    if (st /= 0) call fatal
    call pack_connectivity(offp, idxp)
    scales = [p2scale, p3scale, p4scale, p5scale, p2iscale, p3iscale, p4iscale, p5iscale, &
              d1scale, d2scale, d3scale, d4scale, u1scale, u2scale, u3scale, u4scale]
    st = c_set_connectivity(ctx, c_loc(offp), c_loc(idxp), c_loc(scales))
    if (st /= 0) call fatal
    mscales = [m2scale, m3scale, m4scale, m5scale]
    st = c_set_mpole_scales(ctx, c_loc(mscales))
    if (st /= 0) call fatal
    call set_frames()
    if (use_vdw) call set_vdw()
  end subroutine

  ! vdW description from kvdw (jvdw, radmin, epsilon, radmin4, epsilon4,
  ! ired, kred), vdwpot (v2scale..v5scale, ghal, dhal) and cutoff (vdwcut,
  ! vdwtaper, already absolute after cutoffs.f:241)
  subroutine set_vdw()
    use atoms, only: n
    use vdw, only: jvdw, radmin, epsilon, radmin4, epsilon4, ired, kred
    use vdwpot, only: v2scale, v3scale, v4scale, v5scale, ghal, dhal
    use cutoff, only: vdwcut, vdwtaper
    integer(c_int), allocatable, target :: cl(:), ir(:)
    real(c_double), allocatable, target :: tab(:,:,:), kr(:)
    real(c_double), target :: vs(4)
    integer :: i, nc, st
    nc = size(radmin, 1)
    allocate(cl(n), ir(n), kr(n), tab(nc, nc, 4))
    do i = 1, n
      cl(i) = jvdw(i) - 1
      ir(i) = ired(i) - 1
      kr(i) = kred(i)
    end do
    tab(:,:,1) = radmin
    tab(:,:,2) = epsilon
    tab(:,:,3) = radmin4
    tab(:,:,4) = epsilon4
    vs = [v2scale, v3scale, v4scale, v5scale]
    st = c_set_vdw(ctx, c_loc(cl), int(nc, c_int), c_loc(tab), c_loc(ir), c_loc(kr), c_loc(vs), &
                   vdwcut, vdwtaper, ghal, dhal)
    if (st /= 0) call fatal
  end subroutine

  ! frame atoms for the torques (and rotpole on the device): mpole::pole,
  ! zaxis, xaxis, polaxe ('Z-then-X' -> 1, 'Bisector' -> 2), 0-based atoms
  subroutine set_frames()
    use atoms, only: n
    use mpole, only: pole, zaxis, xaxis, polaxe
    real(c_double), allocatable, target :: pl(:,:)
    integer(c_int), allocatable, target :: zx(:), xx(:), ax(:)
    integer :: i, st
    allocate(pl(13,n), zx(n), xx(n), ax(n))
    do i = 1, n  ! every atom carries a multipole in the water workloads
      pl(:,i) = pole(:,i)
      zx(i) = zaxis(i) - 1
      xx(i) = xaxis(i) - 1
      ax(i) = merge(2, 1, polaxe(i) == 'Bisector')
    end do
    st = c_set_frames(ctx, c_loc(pl), c_loc(zx), c_loc(xx), c_loc(ax))
    if (st /= 0) call fatal
  end subroutine

  ! CSR copies (0-based) of couple::i12..i15 and polgrp::ip11..ip14
  subroutine pack_connectivity(offp, idxp)
    use atoms, only: n
    use couple, only: n12, i12, n13, i13, n14, i14, n15, i15
    use polgrp, only: np11, ip11, np12, ip12, np13, ip13, np14, ip14
    type(c_ptr), intent(out) :: offp(8), idxp(8)
    integer :: s, i, j, m, cap
    cap = max(size(i12,1), size(i13,1), size(i14,1), size(i15,1), size(ip11,1), size(ip12,1), &
              size(ip13,1), size(ip14,1))
    if (allocated(off)) deallocate(off, idx)
    allocate(off(n+1,8), idx(cap*n,8))
    do s = 1, 8
      off(1,s) = 0
      m = 0
      do i = 1, n
        do j = 1, count_of(s, i)
          m = m + 1
          idx(m,s) = entry_of(s, j, i) - 1
        end do
        off(i+1,s) = m
      end do
      offp(s) = c_loc(off(1,s))
      idxp(s) = c_loc(idx(1,s))
    end do
  contains
    integer function count_of(s, i)
      integer, intent(in) :: s, i
      select case (s)
      case (1); count_of = n12(i)
      case (2); count_of = n13(i)
      case (3); count_of = n14(i)
      case (4); count_of = n15(i)
      case (5); count_of = np11(i)
      case (6); count_of = np12(i)
      case (7); count_of = np13(i)
      case default; count_of = np14(i)
      end select
    end function
    integer function entry_of(s, j, i)
      integer, intent(in) :: s, j, i
      select case (s)
      case (1); entry_of = i12(j,i)
      case (2); entry_of = i13(j,i)
      case (3); entry_of = i14(j,i)
      case (4); entry_of = i15(j,i)
      case (5); entry_of = ip11(j,i)
      case (6); entry_of = ip12(j,i)
      case (7); entry_of = ip13(j,i)
      case default; entry_of = ip14(j,i)
      end select
    end function
  end subroutine

  subroutine bind_all()
    use atoms, only: x, y, z
    use mpole, only: rpole
    use polar, only: uind, uinp
    use neigh, only: nelst, elst
    use sizes, only: maxelst
    use energi, only: ep
    integer :: st
    st = c_bind_state(ctx, x, y, z, rpole, uind, uinp, nelst, elst, int(maxelst, c_int), ep)
    if (st /= 0) call fatal
  end subroutine

  subroutine thp_newinduce_pme2
    call bind_all()
    call c_newinduce_pme2()
    if (c_last_error() /= 0 .and. c_last_error() /= 3) call fatal
  end subroutine

  subroutine thp_mlistcell
    call bind_all()
    call c_mlistcell()
    if (c_last_error() /= 0) call fatal
  end subroutine

  subroutine thp_epolar
    call bind_all()
    call c_epolar()
    if (c_last_error() /= 0 .and. c_last_error() /= 3) call fatal
  end subroutine

  ! epolar1 (gradient.f:165): energy into ep, gradient into deriv::dep
  subroutine thp_epolar1
    use deriv, only: dep
    integer :: st
    call bind_all()
    st = c_bind_gradient(ctx, dep)
    if (st /= 0) call fatal
    call c_epolar1()
    if (c_last_error() /= 0 .and. c_last_error() /= 3) call fatal
  end subroutine

  ! empole1 (empole1.f:10): energy into em, gradient into deriv::dem
  ! (overwritten, as empole1c zeroes it)
  subroutine thp_empole1
    use deriv, only: dem
    use energi, only: em
    integer :: st
    call bind_all()
    st = c_bind_mpole(ctx, em, dem)
    if (st /= 0) call fatal
    call c_empole1()
    if (c_last_error() /= 0) call fatal
  end subroutine

  ! ehal1 (ehal1.f:17): energy into ev, gradient into deriv::dev; the vdW
  ! description comes from thp_set_vdw (classes, combined pair tables and
  ! reduction from the kvdw module), set once after kvdw
  subroutine thp_ehal1
    use deriv, only: dev
    use energi, only: ev
    integer :: st
    call bind_all()
    st = c_bind_vdw(ctx, ev, dev)
    if (st /= 0) call fatal
    call c_ehal1()
    if (c_last_error() /= 0) call fatal
  end subroutine

  ! grid_uind_site over a whole site list (pmestuff.f:280), one rank
  subroutine thp_grid_uind_sites(ns, isite, fuind, fuinp, qgrid)
    integer, intent(in) :: ns, isite(ns)
    real*8, intent(in) :: fuind(3,ns), fuinp(3,ns)
    real*8, intent(inout) :: qgrid(*)
    integer(c_int), allocatable :: s(:)
    call bind_all()
    s = int(isite, c_int)
    call c_grid_uind_sites(int(ns, c_int), s, fuind, fuinp, qgrid)
    if (c_last_error() /= 0) call fatal
  end subroutine

  ! fphi_uind_site over a whole site list (pmestuff.f:746), one rank
  subroutine thp_fphi_uind_sites(ns, isite, qgrid, phi1, phi2, sphi)
    integer, intent(in) :: ns, isite(ns)
    real*8, intent(in) :: qgrid(*)
    real*8, intent(out) :: phi1(10,ns), phi2(10,ns), sphi(20,ns)
    integer(c_int), allocatable :: s(:)
    call bind_all()
    s = int(isite, c_int)
    call c_fphi_uind_sites(int(ns, c_int), s, qgrid, phi1, phi2, sphi)
    if (c_last_error() /= 0) call fatal
  end subroutine

  subroutine thp_finalize
    integer :: st
    if (c_associated(ctx)) st = c_ctx_destroy(ctx)
    ctx = c_null_ptr
  end subroutine
end module thp_shim
