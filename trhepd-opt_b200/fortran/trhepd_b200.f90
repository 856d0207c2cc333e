!*******************************************************************
! ISO_C_BINDING interface to libtrhepd_b200.so (include/trhepd_b200.h)
! and a drop-in replacement of srfref for sim-trhepd-rheed.
!
! srfref_b200 keeps srfref's argument list (sim-trhepd-rheed/src/surflf.f90:7-8)
! and its I/O: it reads the bulk reflection records from unit 1 in the same
! order (surflf.f90:65-72), solves every (azimuth, glancing angle) on the GPU in
! one batch, and writes unit 3 with the reference's format (surflf.f90:154-165).
! The mod_scpot3 state (surfio.f90:18-41) is passed by address.
!
! Build:  gfortran -c trhepd_b200.f90 (after mod_scpot3 is compiled), link with
!         -L<dir> -ltrhepd_b200 -lcudart.  In surfio.f90:340 call srfref_b200
!         in place of srfref.
!*******************************************************************
module trhepd_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: TRHEPD_FP64 = 0, TRHEPD_SPLIT_BF16 = 1

  type, bind(C) :: trhepd_pot_state
    integer(c_int) :: nv, nvb, natms, natmb, nelm, nabr, nabi
    type(c_ptr) :: ielm
    real(c_double) :: cc, smesh
    type(c_ptr) :: z, dchg, Ghk, ocr, b, asf, st0, st1, st2
  end type

  interface
    integer(c_int) function trhepd_create(device, ctx) bind(C, name="trhepd_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr) :: ctx
    end function
    subroutine trhepd_destroy(ctx) bind(C, name="trhepd_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine
    integer(c_int) function trhepd_srfref(ctx, pot, nb, ns, iv, dz, ngr, nbg, iord, ih, ik, &
        wn, ghx, ghy, gky, azi, daz, naz, gi, dg, ng, int_method, t1, precision, f2, angle) &
        bind(C, name="trhepd_srfref")
      import :: c_int, c_ptr, c_double, trhepd_pot_state
      type(c_ptr), value :: ctx
      type(trhepd_pot_state), intent(in) :: pot
      integer(c_int), value :: nb, ns, ngr, naz, ng, int_method, precision
      integer(c_int), intent(in) :: iv(nb, nb), nbg(ngr), iord(nb), ih(nb), ik(nb)
      real(c_double), value :: dz, wn, ghx, ghy, gky, azi, daz, gi, dg
      complex(c_double_complex), intent(in) :: t1(*)
      real(c_double), intent(out) :: f2(nb, *), angle(*)
    end function
  end interface

  type(c_ptr), save :: ctx = c_null_ptr

contains

  subroutine srfref_b200(nv,nb,ns,iv,dz,ngr,nbg,iord,ih,ik &
                ,wn,ghx,ghy,gky,azi,daz,naz,gi,dg,ng,idiag,iprn,int_method)
    use mod_scpot3
    implicit none
    real(8) :: dz,wn,ghx,ghy,gky,azi,daz,gi,dg
    integer :: iv(nb,nb),ih(nb),ik(nb),iord(nb),nbg(ngr)
    integer :: nv,nb,ns,ngr,naz,ng,idiag,iprn,int_method

    type(trhepd_pot_state), target :: pot
    complex(8), allocatable, target :: t1(:)
    real(8), allocatable :: f2(:,:), angle(:)
    integer :: nrep1, nrep2, irep1, irep2, l, ib, per, rc, nrec, i, j, o

    if (.not. c_associated(ctx)) then
      rc = trhepd_create(0_c_int, ctx)
      if (rc /= 0) stop 'trhepd_create failed'
    endif
    if (ng > naz) then
      nrep1 = naz; nrep2 = ng
    else
      nrep1 = ng; nrep2 = naz
    endif
    per = 0
    do l = 1, ngr
      per = per + nbg(l)*nbg(l)
    end do
    nrec = nrep1*nrep2
    allocate(t1(per*nrec), f2(nb, nrec), angle(nrec))
    ! bulk reflection records, same order as surflf.f90:65-72
    o = 0
    do irep1 = 1, nrep1
      do irep2 = 1, nrep2
        do l = 1, ngr
          read (1) (t1(o+i), i = 1, nbg(l)*nbg(l))
          o = o + nbg(l)*nbg(l)
        end do
      end do
    end do
    pot%nv = nv; pot%nvb = nvb; pot%natms = natms; pot%natmb = natmb
    pot%nelm = nelm; pot%nabr = nabr; pot%nabi = nabi
    pot%ielm = c_loc(ielm); pot%cc = cc; pot%smesh = smesh
    pot%z = c_loc(z); pot%dchg = c_loc(dchg); pot%Ghk = c_loc(Ghk); pot%ocr = c_loc(ocr)
    pot%b = c_loc(b); pot%asf = c_loc(asf)
    pot%st0 = c_loc(st0); pot%st1 = c_loc(st1); pot%st2 = c_loc(st2)
    rc = trhepd_srfref(ctx, pot, nb, ns, iv, dz, ngr, nbg, iord, ih, ik, wn, ghx, ghy, gky, &
                       azi, daz, naz, gi, dg, ng, int_method, t1, TRHEPD_FP64, f2, angle)
    if (rc /= 0) stop 'trhepd_srfref failed'
    ib = 0
    do irep1 = 1, nrep1
      do irep2 = 1, nrep2
        ib = ib + 1
        write (3,'(E12.4,200(",",E23.15))') angle(ib),(f2(j,ib),j=1,nb)
      end do
      write (3,*)
    end do
    deallocate(t1, f2, angle)
  end subroutine
end module
