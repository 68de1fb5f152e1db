!-----7--------------------------------------------------------------7--
! m_cress_gpu: ISO_C_BINDING interface of the cress_b200 C-ABI
! (include/cress_b200.h) for the CReSS solver.
!
! The reference's hot-path routines are module procedures that take
! name-table ids and explicit-shape arrays a(0:ni+1,0:nj+1,1:nk).  This
! module declares the C entry points with matching Fortran dummies: a
! real(c_float) array in that shape is passed by reference, which is the
! C "const float*" of the same layout (x fastest, halo 0..ni+1, k from 1).
! The derived type cress_cfg mirrors the C struct field by field.
!
! s_intgdrv_gpu shows the body a maintainer puts in place of s_intgdrv
! (SrcOrig/intgdrv.f90:111-1133) for the supported options: the state lives
! on the device between calls; cress_get_field brings a level back before a
! dump or restart write (SrcOrig/outdmp3d.f90, SrcOrig/outres.f90), and
! cress_put_field sends it after a restart read.
!
! No Fortran compiler exists in the build image, so this file is shipped
! as source and checked only by reading; the same calls are exercised from
! C/Python through the identical C-ABI in the test suite.
!-----7--------------------------------------------------------------7--

      module m_cress_gpu

      use iso_c_binding

      implicit none

      integer(c_int), parameter :: cress_ok = 0

      integer(c_int), parameter :: cress_u = 0, cress_v = 1, cress_w = 2
      integer(c_int), parameter :: cress_pp = 3, cress_ptp = 4
      integer(c_int), parameter :: cress_qv = 5, cress_qc = 6, cress_qr = 7
      integer(c_int), parameter :: cress_qi = 8, cress_qs = 9, cress_qg = 10
      integer(c_int), parameter :: cress_ni = 11, cress_ns = 12
      integer(c_int), parameter :: cress_ng = 13, cress_tke = 14

      integer(c_int), parameter :: cress_past = 0, cress_now = 1
      integer(c_int), parameter :: cress_future = 2, cress_forcing = 3

      type, bind(c) :: cress_cfg
        integer(c_int) :: ni, nj, nk
        real(c_float) :: dx, dy, dz
        integer(c_int) :: sthopt, impopt, divopt, buyopt, gwmopt
        real(c_float) :: weicoe
        integer(c_int) :: wbc, ebc, sbc, nbc, bbc, tbc
        integer(c_int) :: tile
        integer(c_int) :: advopt, smtopt, vspopt, coropt, tubopt, cphopt
        real(c_float) :: smhcoe, smvcoe, filcoe, fc
        character(kind=c_char) :: vspvar(16)
        real(c_float) :: thresq
        real(c_float) :: gwave
        integer(c_int) :: reserved(6)
      end type cress_cfg

      interface

        integer(c_int) function cress_create(cfg, device, ctx)          &
     &    bind(c, name='cress_create')
          import :: c_int, c_ptr, cress_cfg
          type(cress_cfg), intent(in) :: cfg
          integer(c_int), value :: device
          type(c_ptr), intent(out) :: ctx
        end function cress_create

        subroutine cress_destroy(ctx) bind(c, name='cress_destroy')
          import :: c_ptr
          type(c_ptr), value :: ctx
        end subroutine cress_destroy

        integer(c_int) function cress_set_base3d(ctx, base3d)           &
     &    bind(c, name='cress_set_base3d')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
          type(c_ptr), intent(in) :: base3d(11)
        end function cress_set_base3d

        integer(c_int) function cress_set_base_large(ctx, ubr, vbr,     &
     &    rbct, ksp0) bind(c, name='cress_set_base_large')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          real(c_float), intent(in) :: ubr(*), vbr(*), rbct(*)
          integer(c_int), value :: ksp0
        end function cress_set_base_large

        integer(c_int) function cress_set_base_moist(ctx, pbr, qvbr)    &
     &    bind(c, name='cress_set_base_moist')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          real(c_float), intent(in) :: pbr(*), qvbr(*)
        end function cress_set_base_moist

        integer(c_int) function cress_put_field(ctx, field, level, a)   &
     &    bind(c, name='cress_put_field')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          integer(c_int), value :: field, level
          real(c_float), intent(in) :: a(*)
        end function cress_put_field

        integer(c_int) function cress_get_field(ctx, field, level, a)   &
     &    bind(c, name='cress_get_field')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          integer(c_int), value :: field, level
          real(c_float), intent(out) :: a(*)
        end function cress_get_field

        integer(c_int) function cress_smalldrv(ctx, nsstp, dts, up, vp, &
     &    wp, ppp, ufrc, vfrc, wfrc, pfrc, uf, vf, wf, ppf)              &
     &    bind(c, name='cress_smalldrv')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          integer(c_int), value :: nsstp
          real(c_float), value :: dts
          real(c_float), intent(in) :: up(*), vp(*), wp(*), ppp(*)
          real(c_float), intent(in) :: ufrc(*), vfrc(*), wfrc(*)
          real(c_float), intent(in) :: pfrc(*)
          real(c_float), intent(out) :: uf(*), vf(*), wf(*), ppf(*)
        end function cress_smalldrv

        integer(c_int) function cress_large_step(ctx, ctime, dtb,       &
     &    nsstp, dts) bind(c, name='cress_large_step')
          import :: c_int, c_ptr, c_float, c_long_long
          type(c_ptr), value :: ctx
          integer(c_long_long), value :: ctime
          real(c_float), value :: dtb
          integer(c_int), value :: nsstp
          real(c_float), value :: dts
        end function cress_large_step

        integer(c_int) function cress_get_precip(ctx, prec)             &
     &    bind(c, name='cress_get_precip')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          real(c_float), intent(out) :: prec(*)
        end function cress_get_precip

        integer(c_int) function cress_get_phase(ctx, field, cpx)       &
     &    bind(c, name='cress_get_phase')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          integer(c_int), value :: field
          real(c_float), intent(out) :: cpx(*)
        end function cress_get_phase

        integer(c_int) function cress_put_phase(ctx, field, cpx)       &
     &    bind(c, name='cress_put_phase')
          import :: c_int, c_ptr, c_float
          type(c_ptr), value :: ctx
          integer(c_int), value :: field
          real(c_float), intent(in) :: cpx(*)
        end function cress_put_phase

! The 1-D base state from a sounding, FP64 on the device (set1d, setbase,
! baserho, sndwave).  sounding(nlev,5): height, u, v, theta or T, and
! relative humidity or mixing ratio; columns(0:nk,11) in the order of the
! C enum cress_base_col (ubr, vbr, pbr, ptbr, qvbr, rbr, ptvbr, pibr, rst,
! rst8w, rcsq).  tvar and hvar are the characters of the reference's
! sndtyp ('p'/'t', 'r'/'q') as c_int codes (ichar).
        integer(c_int) function cress_base_state(nk, zph, jcb, nlev,    &
     &    sounding, tvar, hvar, psnd0, thresq, columns, device)          &
     &    bind(c, name='cress_base_state')
          import :: c_int, c_double
          integer(c_int), value :: nk, nlev, tvar, hvar, device
          real(c_double), intent(in) :: zph(*), jcb(*), sounding(*)
          real(c_double), value :: psnd0, thresq
          real(c_double), intent(out) :: columns(*)
        end function cress_base_state

! Read-back of several fields of one level on a second stream; the host
! arrays (fields(i) -> the i-th address in host) are filled once
! cress_wait_fields returns.  Before a dump (SrcOrig/outdmp3d.f90:159-169).
        integer(c_int) function cress_get_fields_async(ctx, level,      &
     &    nfield, fields, host) bind(c, name='cress_get_fields_async')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int), value :: level, nfield
          integer(c_int), intent(in) :: fields(*)
          type(c_ptr), intent(in) :: host(*)
        end function cress_get_fields_async

        integer(c_int) function cress_wait_fields(ctx)                  &
     &    bind(c, name='cress_wait_fields')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function cress_wait_fields

        integer(c_int) function cress_wait_fields_to(ctx, in_flight)    &
     &    bind(c, name='cress_wait_fields_to')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int), value :: in_flight
        end function cress_wait_fields_to

! Input of several fields of one level on a stream of its own, overlapping
! the work already queued; the host arrays stay unchanged until the next
! synchronizing call.
        integer(c_int) function cress_put_fields_async(ctx, level,      &
     &    nfield, fields, host) bind(c, name='cress_put_fields_async')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
          integer(c_int), value :: level, nfield
          integer(c_int), intent(in) :: fields(*)
          type(c_ptr), intent(in) :: host(*)
        end function cress_put_fields_async

! Dump records of one time level (dmplev = 1, dmpfmt = 2) in the .bin
! file's byte layout; host may be c_null_ptr to query nbytes.  The bytes
! go to the dump file as they are (access='stream', or one direct-access
! record per nx*ny*4 bytes).
        integer(c_int) function cress_dump_3d(ctx, level, dmpvar, host,  &
     &    cap, nbytes, names, ncap) bind(c, name='cress_dump_3d')
          import :: c_int, c_ptr, c_char, c_long_long
          type(c_ptr), value :: ctx, host
          integer(c_int), value :: level, ncap
          character(kind=c_char), intent(in) :: dmpvar(*)
          integer(c_long_long), value :: cap
          integer(c_long_long), intent(out) :: nbytes
          character(kind=c_char), intent(out) :: names(*)
        end function cress_dump_3d

! The device-held restart records, framed as sequential unformatted
! records: written after the base-state records of s_outres (a file opened
! with access='stream' takes them unchanged), read back before s_rdres's.
        integer(c_int) function cress_restart_write(ctx, host, cap,      &
     &    nbytes) bind(c, name='cress_restart_write')
          import :: c_int, c_ptr, c_long_long
          type(c_ptr), value :: ctx, host
          integer(c_long_long), value :: cap
          integer(c_long_long), intent(out) :: nbytes
        end function cress_restart_write

        integer(c_int) function cress_restart_read(ctx, host, nbytes)    &
     &    bind(c, name='cress_restart_read')
          import :: c_int, c_ptr, c_long_long
          type(c_ptr), value :: ctx, host
          integer(c_long_long), value :: nbytes
        end function cress_restart_read

! y-slab decomposition over NCCL (one rank per GPU): id128 from
! cress_slab_nccl_id on one rank, broadcast to all.
        integer(c_int) function cress_slab_nccl_id(id128)                &
     &    bind(c, name='cress_slab_nccl_id')
          import :: c_int, c_ptr
          type(c_ptr), value :: id128
        end function cress_slab_nccl_id

        integer(c_int) function cress_slab_attach_nccl(ctx, rank,        &
     &    nranks, id128) bind(c, name='cress_slab_attach_nccl')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx, id128
          integer(c_int), value :: rank, nranks
        end function cress_slab_attach_nccl

        integer(c_int) function cress_slab_detach(ctx)                  &
     &    bind(c, name='cress_slab_detach')
          import :: c_int, c_ptr
          type(c_ptr), value :: ctx
        end function cress_slab_detach

        type(c_ptr) function cress_last_error()                         &
     &    bind(c, name='cress_last_error')
          import :: c_ptr
        end function cress_last_error

      end interface

      contains

!-----7--------------------------------------------------------------7--

! The body that replaces s_intgdrv for advopt=2 or 3, tubopt=0, 1 or 2, cphopt=0 or 3,
! impopt=1, periodic lateral boundaries, flat terrain: one leapfrog step
! on the device-resident state.  ctime, dtb, nsstp, dts are s_intgdrv's
! own arguments (SrcOrig/intgdrv.f90:111-116).  A nonzero status goes to
! the reference's error path (destroy(...,'stop')).

      subroutine s_intgdrv_gpu(ctx, ctime, dtb, nsstp, dts, stat)

      type(c_ptr), intent(in) :: ctx
      integer(c_long_long), intent(in) :: ctime
      real, intent(in) :: dtb, dts
      integer, intent(in) :: nsstp
      integer, intent(out) :: stat

      stat = cress_large_step(ctx, ctime, real(dtb, c_float),           &
     &                        int(nsstp, c_int), real(dts, c_float))

      end subroutine s_intgdrv_gpu

!-----7--------------------------------------------------------------7--

      end module m_cress_gpu
