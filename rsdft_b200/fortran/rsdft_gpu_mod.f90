!-----------------------------------------------------------------------------
! rsdft_gpu_mod: ISO_C_BINDING interface to librsdft_gpu.so (include/rsdft_gpu.h)
! and thin shims with the call surfaces of RSDFT's eigensolver routines, so a
! Fortran driver swaps the callee and keeps its own code.
!
! Shim                          replaces (RSDFT v1.3.0 src/)
! gpu_hamiltonian               hamiltonian            hamiltonian_module.f90:20
! gpu_conjugate_gradient        conjugate_gradient     cg_module.f90:54
! gpu_gram_schmidt              gram_schmidt           gram_schmidt_module.f90:28
! gpu_subspace_diag             subspace_diag          subspace_diag_module.f90:17
! gpu_subspace_mate_sl          subspace_mate_sl       subspace_mate_sl_module.f90:27
! gpu_subspace_solv_sl          subspace_solv_sl       subspace_solv_sl_module.f90:15
! gpu_subspace_rotv_sl          subspace_rotv_sl       subspace_rotv_sl_module.f90:24
! gpu_calc_sweep                calc_sweep (loop)      sweep_module.f90:60
! gpu_esp_calc                  esp_calc               esp_calc_module.f90:15
! gpu_calc_force_ps_nloc2       calc_force_ps_nloc2    ps_nloc2_module.f90:1281
! gpu_calc_density              calc_density (NCPP)    density_module.f90:115
! gpu_wf_io_write               simple_wf_io_write     io_write_module.f90:19
! gpu_wf_io_read                simple_wf_io_read      io_read_module.f90:15
!
! Grid split over comm_grid / comm_band (one rank per GPU; the driver keeps
! its own MPI for the halo planes, the all-reduces and the all-to-alls):
! gpu_op_local                  op_kinetic + op_localpot on a rank's planes   hamiltonian_module.f90:42,50
! gpu_op_nonlocal_project       op_ps_nloc2_hp partial projections           ps_nloc2_op_module.f90:161-175
! gpu_op_nonlocal_add           op_ps_nloc2_hp scatter                       ps_nloc2_op_module.f90:255-263
! gpu_gram                      the dgemm / dsyr2k partial sums              gram_schmidt_t_module.f90:187,
!                                                                            subspace_diag_la_module.f90:96
! gpu_overlap_cholesky          Cholesky of the summed overlap
! gpu_rr_reduced                reduced eigenproblem, rotation matrix        subspace_diag_la_module.f90:122-200
! gpu_rotate                    subspace_rotv_sl on a rank's own rows        subspace_rotv_sl_module.f90:92
!
! Real Gamma-point build only (-D_DRSDFT_), one MPI rank per GPU.  Arrays are
! passed by address (c_loc); a non-zero status stops the program with the
! library's message, the reference's own convention for fatal errors.
!-----------------------------------------------------------------------------
MODULE rsdft_gpu_mod

  use iso_c_binding

  implicit none

  PRIVATE
  PUBLIC :: gpu_init, gpu_setup_grid, gpu_setup_vloc, gpu_setup_nonlocal, gpu_register_wf, gpu_sync_to_host, &
            gpu_sync_to_device, gpu_hamiltonian, gpu_conjugate_gradient, gpu_gram_schmidt, gpu_subspace_diag, &
            gpu_subspace_mate_sl, gpu_subspace_solv_sl, gpu_subspace_rotv_sl, gpu_esp_calc, gpu_calc_force_ps_nloc2, &
            gpu_calc_density, gpu_wf_io_write, gpu_wf_io_read, gpu_calc_sweep, gpu_op_local, &
            gpu_op_nonlocal_project, gpu_op_nonlocal_add, gpu_gram, gpu_overlap_cholesky, gpu_rr_reduced, gpu_rotate, &
            gpu_write_vrho, gpu_read_vrho

  integer(c_int), parameter, PUBLIC :: RSDFT_MODE_FP64 = 0, RSDFT_MODE_MIXED_BF16X3 = 1, &
                                       RSDFT_MODE_MIXED_TF32 = 2, RSDFT_MODE_MIXED_BF16X2 = 3

  interface
     integer(c_int) function rsdft_gpu_init(device) bind(C, name="rsdft_gpu_init")
       import :: c_int
       integer(c_int), value :: device
     end function rsdft_gpu_init
     type(c_ptr) function rsdft_gpu_last_error() bind(C, name="rsdft_gpu_last_error")
       import :: c_ptr
     end function rsdft_gpu_last_error
     integer(c_int) function rsdft_gpu_set_grid(ngrid, md, coef_lap0, coef_lap, hgrid, ggg, dv) &
          bind(C, name="rsdft_gpu_set_grid")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: ngrid, coef_lap, hgrid, ggg
       integer(c_int), value :: md
       real(c_double), value :: coef_lap0, dv
     end function rsdft_gpu_set_grid
     integer(c_int) function rsdft_gpu_set_vloc(vloc, ml, nspin) bind(C, name="rsdft_gpu_set_vloc")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: vloc
       integer(c_long), value :: ml
       integer(c_int), value :: nspin
     end function rsdft_gpu_set_vloc
     integer(c_int) function rsdft_gpu_set_nonlocal(nzlma, lma_ptr, jjp, uv, iuv, amap, natom, duvdr) &
          bind(C, name="rsdft_gpu_set_nonlocal")
       import :: c_int, c_ptr
       integer(c_int), value :: nzlma, natom
       type(c_ptr), value :: lma_ptr, jjp, uv, iuv, amap, duvdr
     end function rsdft_gpu_set_nonlocal
     integer(c_int) function rsdft_gpu_register_wf(unk, ml, mb) bind(C, name="rsdft_gpu_register_wf")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: unk
       integer(c_long), value :: ml
       integer(c_int), value :: mb
     end function rsdft_gpu_register_wf
     integer(c_int) function rsdft_gpu_sync_to_host(unk) bind(C, name="rsdft_gpu_sync_to_host")
       import :: c_int, c_ptr
       type(c_ptr), value :: unk
     end function rsdft_gpu_sync_to_host
     integer(c_int) function rsdft_gpu_sync_to_device(unk) bind(C, name="rsdft_gpu_sync_to_device")
       import :: c_int, c_ptr
       type(c_ptr), value :: unk
     end function rsdft_gpu_sync_to_device
     integer(c_int) function rsdft_gpu_hamiltonian(k, s, tpsi, htpsi, n1, n2, ib1, ib2) &
          bind(C, name="rsdft_gpu_hamiltonian")
       import :: c_int, c_ptr
       integer(c_int), value :: k, s, n1, n2, ib1, ib2
       type(c_ptr), value :: tpsi, htpsi
     end function rsdft_gpu_hamiltonian
     integer(c_int) function rsdft_gpu_conjugate_gradient(n1, n2, mb, k, s, unk, esp, res, ncg, mloop, ipc, mode) &
          bind(C, name="rsdft_gpu_conjugate_gradient")
       import :: c_int, c_ptr
       integer(c_int), value :: n1, n2, mb, k, s, ncg, mloop, ipc, mode
       type(c_ptr), value :: unk, esp, res
     end function rsdft_gpu_conjugate_gradient
     integer(c_int) function rsdft_gpu_gram_schmidt(n0, n1, k, s, unk, ld, nblk, nblk1, mode) &
          bind(C, name="rsdft_gpu_gram_schmidt")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: n0, n1, k, s, nblk, nblk1, mode
       type(c_ptr), value :: unk
       integer(c_long), value :: ld
     end function rsdft_gpu_gram_schmidt
     integer(c_int) function rsdft_gpu_subspace_diag(k, s, unk, ld, mb, esp, mode) &
          bind(C, name="rsdft_gpu_subspace_diag")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: k, s, mb, mode
       type(c_ptr), value :: unk, esp
       integer(c_long), value :: ld
     end function rsdft_gpu_subspace_diag
     integer(c_int) function rsdft_gpu_orth_subspace_diag(k, s, unk, ld, mb, esp, mode) &
          bind(C, name="rsdft_gpu_orth_subspace_diag")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: k, s, mb, mode
       type(c_ptr), value :: unk, esp
       integer(c_long), value :: ld
     end function rsdft_gpu_orth_subspace_diag
     integer(c_int) function rsdft_gpu_eigensolver_sweep(k, s, unk, ld, mb, esp, res, ncg, mloop, ipc, mode) &
          bind(C, name="rsdft_gpu_eigensolver_sweep")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: k, s, mb, ncg, mloop, ipc, mode
       type(c_ptr), value :: unk, esp, res
       integer(c_long), value :: ld
     end function rsdft_gpu_eigensolver_sweep
     integer(c_int) function rsdft_gpu_calc_sweep(unk, ld, mb, nspin, esp, res, occ, diter, iconv_check, tol_esp, &
          mb_ref, nelectron, nfixed, dspn, ekbt, kinteg, ncg, mloop, ipc, mode, iter_out, conv_out, efermi) &
          bind(C, name="rsdft_gpu_calc_sweep")
       import :: c_int, c_long, c_double, c_ptr
       type(c_ptr), value :: unk, esp, res, occ, iter_out, conv_out, efermi
       integer(c_long), value :: ld
       integer(c_int), value :: mb, nspin, diter, iconv_check, mb_ref, nfixed, kinteg, ncg, mloop, ipc, mode
       real(c_double), value :: tol_esp, nelectron, dspn, ekbt
     end function rsdft_gpu_calc_sweep
     integer(c_int) function rsdft_gpu_subspace_mate(k, s, unk, ld, mb, hsub, ldh) &
          bind(C, name="rsdft_gpu_subspace_mate")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: k, s, mb, ldh
       type(c_ptr), value :: unk, hsub
       integer(c_long), value :: ld
     end function rsdft_gpu_subspace_mate
     integer(c_int) function rsdft_gpu_subspace_solv(mb, hsub, ldh, esp, vsub, ldv) &
          bind(C, name="rsdft_gpu_subspace_solv")
       import :: c_int, c_ptr
       integer(c_int), value :: mb, ldh, ldv
       type(c_ptr), value :: hsub, esp, vsub
     end function rsdft_gpu_subspace_solv
     integer(c_int) function rsdft_gpu_subspace_rotv(k, s, unk, ld, mb, vsub, ldv) &
          bind(C, name="rsdft_gpu_subspace_rotv")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: k, s, mb, ldv
       type(c_ptr), value :: unk, vsub
       integer(c_long), value :: ld
     end function rsdft_gpu_subspace_rotv
     integer(c_int) function rsdft_gpu_esp_calc(k, s, wf, n1, n2, ns, ne, e) bind(C, name="rsdft_gpu_esp_calc")
       import :: c_int, c_ptr
       integer(c_int), value :: k, s, n1, n2, ns, ne
       type(c_ptr), value :: wf, e
     end function rsdft_gpu_esp_calc
     integer(c_int) function rsdft_gpu_force_nloc(mi, unk, ld, mb, occ, force2) bind(C, name="rsdft_gpu_force_nloc")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: mi, mb
       type(c_ptr), value :: unk, occ, force2
       integer(c_long), value :: ld
     end function rsdft_gpu_force_nloc
     integer(c_int) function rsdft_gpu_calc_density(unk, ld, mb, occ, rho) bind(C, name="rsdft_gpu_calc_density")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: unk, occ, rho
       integer(c_long), value :: ld
       integer(c_int), value :: mb
     end function rsdft_gpu_calc_density
     integer(c_int) function rsdft_gpu_write_wf(path, unk, ld, mb, mk, ms, mbwr1, mbwr2, oc, io_ctrl, ngrid, occ, &
          aa, bb, mmbz, kbb) bind(C, name="rsdft_gpu_write_wf")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: path, unk, ngrid, occ, aa, bb, kbb
       integer(c_long), value :: ld
       integer(c_int), value :: mb, mk, ms, mbwr1, mbwr2, oc, io_ctrl, mmbz
     end function rsdft_gpu_write_wf
     integer(c_int) function rsdft_gpu_read_wf(path, unk, ld, mb, mk, ms, io_ctrl, ngrid, occ, info) &
          bind(C, name="rsdft_gpu_read_wf")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: path, unk, ngrid, occ, info
       integer(c_long), value :: ld
       integer(c_int), value :: mb, mk, ms, io_ctrl
     end function rsdft_gpu_read_wf
     integer(c_int) function rsdft_gpu_write_vrho(path, ngrid, aa, nelement, natom, aa_atom, ki_atom, zn_atom, &
          efermi, nspin, rho, vloc, vh, vxc) bind(C, name="rsdft_gpu_write_vrho")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: path, ngrid, aa, aa_atom, ki_atom, zn_atom, rho, vloc, vh, vxc
       integer(c_int), value :: nelement, natom, nspin
       real(c_double), value :: efermi
     end function rsdft_gpu_write_vrho
     integer(c_int) function rsdft_gpu_read_vrho(path, ngrid, nspin, rho, vloc, vh, vxc, efermi) &
          bind(C, name="rsdft_gpu_read_vrho")
       import :: c_int, c_ptr
       type(c_ptr), value :: path, ngrid, rho, vloc, vh, vxc, efermi
       integer(c_int), value :: nspin
     end function rsdft_gpu_read_vrho
     integer(c_int) function rsdft_gpu_op_local(s, tpsi, htpsi, ld, nb, z0, nz) bind(C, name="rsdft_gpu_op_local")
       import :: c_int, c_long, c_ptr
       integer(c_int), value :: s, nb, z0, nz
       type(c_ptr), value :: tpsi, htpsi
       integer(c_long), value :: ld
     end function rsdft_gpu_op_local
     integer(c_int) function rsdft_gpu_op_nonlocal_project(tpsi, ld, nb, uvunk) &
          bind(C, name="rsdft_gpu_op_nonlocal_project")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: tpsi, uvunk
       integer(c_long), value :: ld
       integer(c_int), value :: nb
     end function rsdft_gpu_op_nonlocal_project
     integer(c_int) function rsdft_gpu_op_nonlocal_add(uvunk, htpsi, ld, nb) bind(C, name="rsdft_gpu_op_nonlocal_add")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: uvunk, htpsi
       integer(c_long), value :: ld
       integer(c_int), value :: nb
     end function rsdft_gpu_op_nonlocal_add
     integer(c_int) function rsdft_gpu_gram(a, b, ld, rows, m, n, alpha, sym, c, ldc) bind(C, name="rsdft_gpu_gram")
       import :: c_int, c_long, c_double, c_ptr
       type(c_ptr), value :: a, b, c
       integer(c_long), value :: ld, rows
       integer(c_int), value :: m, n, sym, ldc
       real(c_double), value :: alpha
     end function rsdft_gpu_gram
     integer(c_int) function rsdft_gpu_overlap_cholesky(mb, s, lds, rinv, ldr, kappa) &
          bind(C, name="rsdft_gpu_overlap_cholesky")
       import :: c_int, c_ptr
       integer(c_int), value :: mb, lds, ldr
       type(c_ptr), value :: s, rinv, kappa
     end function rsdft_gpu_overlap_cholesky
     integer(c_int) function rsdft_gpu_rr_reduced(mb, rinv, ldr, hsub, ldh, esp, w, ldw) &
          bind(C, name="rsdft_gpu_rr_reduced")
       import :: c_int, c_ptr
       integer(c_int), value :: mb, ldr, ldh, ldw
       type(c_ptr), value :: rinv, hsub, esp, w
     end function rsdft_gpu_rr_reduced
     integer(c_int) function rsdft_gpu_rotate(unk, ld, rows, mb, v, ldv) bind(C, name="rsdft_gpu_rotate")
       import :: c_int, c_long, c_ptr
       type(c_ptr), value :: unk, v
       integer(c_long), value :: ld, rows
       integer(c_int), value :: mb, ldv
     end function rsdft_gpu_rotate
  end interface

CONTAINS

  SUBROUTINE check(ierr, who)
    integer(c_int), intent(IN) :: ierr
    character(*), intent(IN) :: who
    character(kind=c_char), pointer :: msg(:)
    character(len=1024) :: text
    integer :: i
    if ( ierr == 0 ) return
    call c_f_pointer(rsdft_gpu_last_error(), msg, [1024])
    text = ""
    do i = 1, 1024
       if ( msg(i) == c_null_char ) exit
       text(i:i) = msg(i)
    end do
    write(*,*) "rsdft_gpu: ", who, " status ", ierr, ": ", trim(text)
    stop "rsdft_gpu"
  END SUBROUTINE check

  SUBROUTINE gpu_init(device)
    integer, intent(IN) :: device
    call check(rsdft_gpu_init(int(device, c_int)), "init")
  END SUBROUTINE gpu_init

  ! Ngrid(1:3), Md, coef_lap0, coef_lap(3,Md), Hgrid(1:3), ggg(1:3), dV
  ! (kinetic_variables / rgrid_module after init_kinetic)
  SUBROUTINE gpu_setup_grid(ngrid, md, coef_lap0, coef_lap, hgrid, ggg, dv)
    integer, intent(IN) :: ngrid(3), md
    real(8), intent(IN) :: coef_lap0, dv
    real(8), intent(IN) :: coef_lap(3, md), hgrid(3), ggg(3)
    integer(c_int), target :: ng(3)
    real(c_double), target :: cl(md, 3), h(3), g(3)
    ng = ngrid
    cl = transpose(coef_lap)  ! axis-major: coef_lap[axis*Md + m-1]
    h = hgrid
    g = ggg
    call check(rsdft_gpu_set_grid(c_loc(ng), int(md, c_int), coef_lap0, c_loc(cl), c_loc(h), c_loc(g), dv), &
               "set_grid")
  END SUBROUTINE gpu_setup_grid

  SUBROUTINE gpu_setup_vloc(vloc, ml, nspin)
    integer, intent(IN) :: ml, nspin
    real(8), intent(IN), target :: vloc(ml, nspin)
    call check(rsdft_gpu_set_vloc(c_loc(vloc), int(ml, c_long), int(nspin, c_int)), "set_vloc")
  END SUBROUTINE gpu_setup_vloc

  ! uVk(MAXMJJ,nzlma,1), JJP(MAXMJJ,nzlma), MJJ(nzlma), iuV(nzlma), amap(nzlma)
  ! (ps_nloc2_variables after prep_ps_nloc2) converted to the CSR of the C side.
  SUBROUTINE gpu_setup_nonlocal(nzlma, maxmjj, mjj, jjp, uvk, iuv, amap, natom, duvdr)
    integer, intent(IN) :: nzlma, maxmjj, natom
    integer, intent(IN) :: mjj(nzlma), jjp(maxmjj, nzlma), iuv(nzlma), amap(nzlma)
    real(8), intent(IN) :: uvk(maxmjj, nzlma)
    real(8), intent(IN), optional :: duvdr(3, maxmjj, nzlma)
    integer(c_int), allocatable, target :: ptr(:), jj(:), iu(:), am(:)
    real(c_double), allocatable, target :: uv(:), du(:)
    integer :: lma, j, n, nnz
    nnz = sum(mjj)
    allocate( ptr(nzlma + 1), jj(max(nnz, 1)), uv(max(nnz, 1)), iu(max(nzlma, 1)), am(max(nzlma, 1)) )
    allocate( du(max(3 * nnz, 1)) )
    n = 0
    ptr(1) = 0
    do lma = 1, nzlma
       do j = 1, mjj(lma)
          n = n + 1
          jj(n) = jjp(j, lma) - 1          ! 0-based grid index
          uv(n) = uvk(j, lma)
          if ( present(duvdr) ) du(3 * n - 2:3 * n) = duvdr(:, j, lma)
       end do
       ptr(lma + 1) = n
       iu(lma) = iuv(lma)
       am(lma) = amap(lma) - 1             ! 0-based atom
    end do
    if ( present(duvdr) ) then
       call check(rsdft_gpu_set_nonlocal(int(nzlma, c_int), c_loc(ptr), c_loc(jj), c_loc(uv), c_loc(iu), &
                  c_loc(am), int(natom, c_int), c_loc(du)), "set_nonlocal")
    else
       call check(rsdft_gpu_set_nonlocal(int(nzlma, c_int), c_loc(ptr), c_loc(jj), c_loc(uv), c_loc(iu), &
                  c_loc(am), int(natom, c_int), c_null_ptr), "set_nonlocal")
    end if
    deallocate( du, am, iu, uv, jj, ptr )
  END SUBROUTINE gpu_setup_nonlocal

  SUBROUTINE gpu_register_wf(unk, ml, mb)
    integer, intent(IN) :: ml, mb
    real(8), intent(INOUT), target :: unk(ml, mb)
    call check(rsdft_gpu_register_wf(c_loc(unk), int(ml, c_long), int(mb, c_int)), "register_wf")
  END SUBROUTINE gpu_register_wf

  SUBROUTINE gpu_sync_to_host(unk)
    real(8), intent(INOUT), target :: unk(:, :)
    call check(rsdft_gpu_sync_to_host(c_loc(unk)), "sync_to_host")
  END SUBROUTINE gpu_sync_to_host

  SUBROUTINE gpu_sync_to_device(unk)
    real(8), intent(INOUT), target :: unk(:, :)
    call check(rsdft_gpu_sync_to_device(c_loc(unk)), "sync_to_device")
  END SUBROUTINE gpu_sync_to_device

  SUBROUTINE gpu_hamiltonian(k, s, tpsi, htpsi, n1, n2, ib1, ib2)
    integer, intent(IN) :: k, s, n1, n2, ib1, ib2
    real(8), intent(IN), target :: tpsi(n1:n2, ib1:ib2)
    real(8), intent(OUT), target :: htpsi(n1:n2, ib1:ib2)
    call check(rsdft_gpu_hamiltonian(k, s, c_loc(tpsi), c_loc(htpsi), n1, n2, ib1, ib2), "hamiltonian")
  END SUBROUTINE gpu_hamiltonian

  SUBROUTINE gpu_conjugate_gradient(n1, n2, mb, k, s, unk, esp, res, ncg, mloop, ipc, mode)
    integer, intent(IN) :: n1, n2, mb, k, s, ncg, mloop, ipc, mode
    real(8), intent(INOUT), target :: unk(n1:n2, mb)
    real(8), intent(INOUT), target :: esp(mb), res(mb)
    call check(rsdft_gpu_conjugate_gradient(n1, n2, mb, k, s, c_loc(unk), c_loc(esp), c_loc(res), ncg, mloop, ipc, &
               mode), "conjugate_gradient")
  END SUBROUTINE gpu_conjugate_gradient

  ! Grid split (z planes of a slab extended by Md halo planes either side;
  ! the halo exchange, the uVunk all-reduce and the MB x MB all-reduces are
  ! the driver's MPI).  z0 is 0-based: op_local on the own planes of an
  ! extended slab is z0 = Md, nz = the own plane count.
  SUBROUTINE gpu_op_local(s, tpsi, htpsi, ld, nb, z0, nz)
    integer, intent(IN) :: s, ld, nb, z0, nz
    real(8), intent(IN), target :: tpsi(ld, nb)
    real(8), intent(INOUT), target :: htpsi(ld, nb)
    call check(rsdft_gpu_op_local(int(s, c_int), c_loc(tpsi), c_loc(htpsi), int(ld, c_long), int(nb, c_int), &
               int(z0, c_int), int(nz, c_int)), "op_local")
  END SUBROUTINE gpu_op_local

  SUBROUTINE gpu_op_nonlocal_project(tpsi, ld, nb, uvunk)
    integer, intent(IN) :: ld, nb
    real(8), intent(IN), target :: tpsi(ld, nb)
    real(8), intent(OUT), target :: uvunk(:, :)
    call check(rsdft_gpu_op_nonlocal_project(c_loc(tpsi), int(ld, c_long), int(nb, c_int), c_loc(uvunk)), &
               "op_nonlocal_project")
  END SUBROUTINE gpu_op_nonlocal_project

  SUBROUTINE gpu_op_nonlocal_add(uvunk, htpsi, ld, nb)
    integer, intent(IN) :: ld, nb
    real(8), intent(IN), target :: uvunk(:, :)
    real(8), intent(INOUT), target :: htpsi(ld, nb)
    call check(rsdft_gpu_op_nonlocal_add(c_loc(uvunk), c_loc(htpsi), int(ld, c_long), int(nb, c_int)), &
               "op_nonlocal_add")
  END SUBROUTINE gpu_op_nonlocal_add

  ! c(1:m, 1:n) = alpha a(1:rows, 1:m)^T b(1:rows, 1:n) (sym = 1: the
  ! symmetric part of a square product), the partial sum of a rank's rows
  SUBROUTINE gpu_gram(a, b, ld, rows, m, n, alpha, sym, c)
    integer, intent(IN) :: ld, rows, m, n, sym
    real(8), intent(IN) :: alpha
    real(8), intent(IN), target :: a(ld, m), b(ld, n)
    real(8), intent(OUT), target :: c(m, n)
    call check(rsdft_gpu_gram(c_loc(a), c_loc(b), int(ld, c_long), int(rows, c_long), int(m, c_int), &
               int(n, c_int), alpha, int(sym, c_int), c_loc(c), int(m, c_int)), "gram")
  END SUBROUTINE gpu_gram

  ! s = R^T R, rinv = R^-1 (upper); kappa = (max diag R / min diag R)^2
  SUBROUTINE gpu_overlap_cholesky(mb, s, rinv, kappa)
    integer, intent(IN) :: mb
    real(8), intent(IN), target :: s(mb, mb)
    real(8), intent(OUT), target :: rinv(mb, mb)
    real(8), intent(OUT), target :: kappa
    call check(rsdft_gpu_overlap_cholesky(int(mb, c_int), c_loc(s), int(mb, c_int), c_loc(rinv), int(mb, c_int), &
               c_loc(kappa)), "overlap_cholesky")
  END SUBROUTINE gpu_overlap_cholesky

  ! R^-T hsub R^-1 = V diag(esp) V^T, w = R^-1 V
  SUBROUTINE gpu_rr_reduced(mb, rinv, hsub, esp, w)
    integer, intent(IN) :: mb
    real(8), intent(IN), target :: rinv(mb, mb), hsub(mb, mb)
    real(8), intent(OUT), target :: esp(mb), w(mb, mb)
    call check(rsdft_gpu_rr_reduced(int(mb, c_int), c_loc(rinv), int(mb, c_int), c_loc(hsub), int(mb, c_int), &
               c_loc(esp), c_loc(w), int(mb, c_int)), "rr_reduced")
  END SUBROUTINE gpu_rr_reduced

  ! unk(1:rows, 1:mb) <- unk v on a registered unk (a rank's own rows)
  SUBROUTINE gpu_rotate(unk, ld, rows, mb, v)
    integer, intent(IN) :: ld, rows, mb
    real(8), intent(INOUT), target :: unk(ld, mb)
    real(8), intent(IN), target :: v(mb, mb)
    call check(rsdft_gpu_rotate(c_loc(unk), int(ld, c_long), int(rows, c_long), int(mb, c_int), c_loc(v), &
               int(mb, c_int)), "rotate")
  END SUBROUTINE gpu_rotate

  ! calc_sweep's loop for one Gamma point: unk(ML, MB, nspin) stays on the
  ! device (register it first); esp holds esp0 on entry; ierr_out is the
  ! iteration the loop stopped at, as the reference's (its loop leaves at
  ! iter == Diter at the latest, so its "not converged" -2 never occurs)
  SUBROUTINE gpu_calc_sweep(unk, esp, res, occ, Diter, iconv_check, tol_esp, mb_ref, Nelectron, Nfixed, dspn, &
                            ekbt, kinteg, ncg, mloop, ipc, mode, ierr_out, efermi)
    real(8), intent(INOUT), target :: unk(:, :, :)
    real(8), intent(INOUT), target :: esp(:, :), res(:, :), occ(:, :)
    integer, intent(IN) :: Diter, iconv_check, mb_ref, Nfixed, kinteg, ncg, mloop, ipc, mode
    real(8), intent(IN) :: tol_esp, Nelectron, dspn, ekbt
    integer, intent(OUT) :: ierr_out
    real(8), intent(OUT), target :: efermi
    integer(c_int), target :: it, cv
    call check(rsdft_gpu_calc_sweep(c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               int(size(unk, 3), c_int), c_loc(esp), c_loc(res), c_loc(occ), Diter, iconv_check, tol_esp, mb_ref, &
               Nelectron, Nfixed, dspn, ekbt, kinteg, ncg, mloop, ipc, mode, c_loc(it), c_loc(cv), c_loc(efermi)), &
               "calc_sweep")
    ierr_out = it
  END SUBROUTINE gpu_calc_sweep

  SUBROUTINE gpu_gram_schmidt(n0, n1, k, s, unk, mode)
    integer, intent(IN) :: n0, n1, k, s, mode
    real(8), intent(INOUT), target :: unk(:, :)
    call check(rsdft_gpu_gram_schmidt(n0, n1, k, s, c_loc(unk), int(size(unk, 1), c_long), 0, 4, mode), &
               "gram_schmidt")
  END SUBROUTINE gpu_gram_schmidt

  SUBROUTINE gpu_subspace_diag(k, s, unk, esp, mode)
    integer, intent(IN) :: k, s, mode
    real(8), intent(INOUT), target :: unk(:, :)
    real(8), intent(OUT), target :: esp(:)
    call check(rsdft_gpu_subspace_diag(k, s, c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               c_loc(esp), mode), "subspace_diag")
  END SUBROUTINE gpu_subspace_diag

  ! gram_schmidt + subspace_diag of calc_sweep (sweep_module.f90:152-155) in one
  ! Rayleigh-Ritz step
  SUBROUTINE gpu_orth_subspace_diag(k, s, unk, esp, mode)
    integer, intent(IN) :: k, s, mode
    real(8), intent(INOUT), target :: unk(:, :)
    real(8), intent(OUT), target :: esp(:)
    call check(rsdft_gpu_orth_subspace_diag(k, s, c_loc(unk), int(size(unk, 1), c_long), &
               int(size(unk, 2), c_int), c_loc(esp), mode), "orth_subspace_diag")
  END SUBROUTINE gpu_orth_subspace_diag

  ! one calc_sweep iteration for (k, s) (sweep_module.f90:150-155)
  SUBROUTINE gpu_eigensolver_sweep(k, s, unk, esp, res, ncg, mloop, ipc, mode)
    integer, intent(IN) :: k, s, ncg, mloop, ipc, mode
    real(8), intent(INOUT), target :: unk(:, :)
    real(8), intent(OUT), target :: esp(:), res(:)
    call check(rsdft_gpu_eigensolver_sweep(k, s, c_loc(unk), int(size(unk, 1), c_long), &
               int(size(unk, 2), c_int), c_loc(esp), c_loc(res), ncg, mloop, ipc, mode), "eigensolver_sweep")
  END SUBROUTINE gpu_eigensolver_sweep

  SUBROUTINE gpu_subspace_mate_sl(k, s, unk, hsub)
    integer, intent(IN) :: k, s
    real(8), intent(IN), target :: unk(:, :)
    real(8), intent(OUT), target :: hsub(:, :)
    call check(rsdft_gpu_subspace_mate(k, s, c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               c_loc(hsub), int(size(hsub, 1), c_int)), "subspace_mate_sl")
  END SUBROUTINE gpu_subspace_mate_sl

  SUBROUTINE gpu_subspace_solv_sl(hsub, esp, vsub)
    real(8), intent(IN), target :: hsub(:, :)
    real(8), intent(OUT), target :: esp(:), vsub(:, :)
    call check(rsdft_gpu_subspace_solv(int(size(hsub, 2), c_int), c_loc(hsub), int(size(hsub, 1), c_int), &
               c_loc(esp), c_loc(vsub), int(size(vsub, 1), c_int)), "subspace_solv_sl")
  END SUBROUTINE gpu_subspace_solv_sl

  SUBROUTINE gpu_subspace_rotv_sl(k, s, unk, vsub)
    integer, intent(IN) :: k, s
    real(8), intent(INOUT), target :: unk(:, :)
    real(8), intent(IN), target :: vsub(:, :)
    call check(rsdft_gpu_subspace_rotv(k, s, c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               c_loc(vsub), int(size(vsub, 1), c_int)), "subspace_rotv_sl")
  END SUBROUTINE gpu_subspace_rotv_sl

  SUBROUTINE gpu_esp_calc(k, s, wf, n1, n2, ns, ne, e)
    integer, intent(IN) :: k, s, n1, n2, ns, ne
    real(8), intent(IN), target :: wf(n1:n2, ns:ne)
    real(8), intent(OUT), target :: e(ns:ne)
    call check(rsdft_gpu_esp_calc(k, s, c_loc(wf), n1, n2, ns, ne, c_loc(e)), "esp_calc")
  END SUBROUTINE gpu_esp_calc

  SUBROUTINE gpu_calc_force_ps_nloc2(mi, force2, unk, occ)
    integer, intent(IN) :: mi
    real(8), intent(OUT), target :: force2(3, mi)
    real(8), intent(IN), target :: unk(:, :), occ(:)
    call check(rsdft_gpu_force_nloc(int(mi, c_int), c_loc(unk), int(size(unk, 1), c_long), &
               int(size(unk, 2), c_int), c_loc(occ), c_loc(force2)), "calc_force_ps_nloc2")
  END SUBROUTINE gpu_calc_force_ps_nloc2

  ! calc_density's NCPP branch (density_module.f90:129-136) for one (k, s)
  ! block: rho(:) = sum_n occ(n) unk(:, n)**2
  SUBROUTINE gpu_calc_density(unk, occ, rho)
    real(8), intent(IN), target :: unk(:, :), occ(:)
    real(8), intent(OUT), target :: rho(:)
    call check(rsdft_gpu_calc_density(c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               c_loc(occ), c_loc(rho)), "calc_density")
  END SUBROUTINE gpu_calc_density

  ! file name as a NUL-terminated C string
  SUBROUTINE c_path(file, buf)
    character(*), intent(IN) :: file
    character(kind=c_char), allocatable, intent(OUT) :: buf(:)
    integer :: i, n
    n = len_trim(file)
    allocate( buf(n + 1) )
    do i = 1, n
       buf(i) = file(i:i)
    end do
    buf(n + 1) = c_null_char
  END SUBROUTINE c_path

  ! simple_wf_io_write(file_wf, IO_ctrl, OC, SYStype=0, MBwr1, MBwr2, ...)
  ! (io_write_module.f90:19) for one process, from the device mirror of a
  ! registered unk; Ngrid(1:3), occ, aa, bb, kbb(3,MMBZ) as in the modules
  ! the reference writer reads.
  SUBROUTINE gpu_wf_io_write(file_wf, io_ctrl, oc, mbwr1, mbwr2, unk, ngrid, occ, aa, bb, kbb)
    character(*), intent(IN) :: file_wf
    integer, intent(IN) :: io_ctrl, oc, mbwr1, mbwr2, ngrid(3)
    real(8), intent(IN), target :: unk(:, :, :, :), occ(:, :, :), aa(3, 3), bb(3, 3), kbb(:, :)
    character(kind=c_char), allocatable, target :: cpath(:)
    integer(c_int), target :: ng(3)
    real(c_double), target :: a(3, 3), b(3, 3)
    ng = ngrid
    a = aa
    b = bb
    call c_path(file_wf, cpath)
    call check(rsdft_gpu_write_wf(c_loc(cpath), c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               int(size(unk, 3), c_int), int(size(unk, 4), c_int), int(mbwr1, c_int), int(mbwr2, c_int), &
               int(oc, c_int), int(io_ctrl, c_int), c_loc(ng), c_loc(occ), c_loc(a), c_loc(b), &
               int(size(kbb, 2), c_int), c_loc(kbb)), "wf_io_write")
  END SUBROUTINE gpu_wf_io_write

  ! simple_wf_io_read(file_wf, SYStype=0, IO_ctrl, ...) (io_read_module.f90:15)
  ! for one process, into the device mirror of a registered unk and occ.
  SUBROUTINE gpu_wf_io_read(file_wf, io_ctrl, unk, ngrid, occ)
    character(*), intent(IN) :: file_wf
    integer, intent(IN) :: io_ctrl, ngrid(3)
    real(8), intent(INOUT), target :: unk(:, :, :, :), occ(:, :, :)
    character(kind=c_char), allocatable, target :: cpath(:)
    integer(c_int), target :: ng(3), info(13)
    ng = ngrid
    call c_path(file_wf, cpath)
    call check(rsdft_gpu_read_wf(c_loc(cpath), c_loc(unk), int(size(unk, 1), c_long), int(size(unk, 2), c_int), &
               int(size(unk, 3), c_int), int(size(unk, 4), c_int), int(io_ctrl, c_int), c_loc(ng), c_loc(occ), &
               c_loc(info)), "wf_io_read")
  END SUBROUTINE gpu_wf_io_read

  ! The density/potential branch of write_data (io_module.f90:97-226) for one
  ! process: rho, Vloc, Vxc (ML, MSP) and Vh (ML) from the modules the
  ! reference writer reads (host arrays or registered ones, whose device
  ! mirrors are written), with the lattice, atoms and Fermi energy.
  SUBROUTINE gpu_write_vrho(file_vrho, ngrid, aa, aa_atom, ki_atom, zn_atom, efermi, rho, vloc, vh, vxc)
    character(*), intent(IN) :: file_vrho
    integer, intent(IN) :: ngrid(3), ki_atom(:), zn_atom(:)
    real(8), intent(IN) :: aa(3, 3), efermi
    real(8), intent(IN), target :: aa_atom(:, :), rho(:, :), vloc(:, :), vh(:), vxc(:, :)
    character(kind=c_char), allocatable, target :: cpath(:)
    integer(c_int), target :: ng(3)
    integer(c_int), allocatable, target :: ki(:), zn(:)
    real(c_double), target :: a(3, 3)
    ng = ngrid
    a = aa
    ki = ki_atom
    zn = zn_atom
    call c_path(file_vrho, cpath)
    call check(rsdft_gpu_write_vrho(c_loc(cpath), c_loc(ng), c_loc(a), int(size(zn), c_int), int(size(ki), c_int), &
               c_loc(aa_atom), c_loc(ki), c_loc(zn), real(efermi, c_double), int(size(rho, 2), c_int), &
               c_loc(rho), c_loc(vloc), c_loc(vh), c_loc(vxc)), "write_vrho")
  END SUBROUTINE gpu_write_vrho

  ! The VRHO branch of read_data (io_module.f90:283-432) for one process:
  ! fills rho, Vloc, Vxc (ML, MSP) and Vh (ML) through the file's LL2 map;
  ! efermi is set from a versioned file and left as it is otherwise.
  SUBROUTINE gpu_read_vrho(file_vrho, ngrid, rho, vloc, vh, vxc, efermi)
    character(*), intent(IN) :: file_vrho
    integer, intent(IN) :: ngrid(3)
    real(8), intent(INOUT), target :: rho(:, :), vloc(:, :), vh(:), vxc(:, :)
    real(8), intent(INOUT), target :: efermi
    character(kind=c_char), allocatable, target :: cpath(:)
    integer(c_int), target :: ng(3)
    ng = ngrid
    call c_path(file_vrho, cpath)
    call check(rsdft_gpu_read_vrho(c_loc(cpath), c_loc(ng), int(size(rho, 2), c_int), c_loc(rho), c_loc(vloc), &
               c_loc(vh), c_loc(vxc), c_loc(efermi)), "read_vrho")
  END SUBROUTINE gpu_read_vrho

END MODULE rsdft_gpu_mod
