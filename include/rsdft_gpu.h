/*
 * rsdft_gpu.h - C ABI of the B200 (sm_100a) Kohn-Sham eigensolver inner loop.
 *
 * Drop-in for the real Gamma-point (-D_DRSDFT_) call surfaces of RSDFT
 * (j-iwata/RSDFT v1.3.0, paths relative to its src/ directory).  The Fortran
 * side binds these with ISO_C_BINDING (bind(C), scalars by value, arrays as
 * plain addresses); every entry returns an int status (0 = OK, < 0 = error,
 * detail in rsdft_gpu_last_error()).
 *
 * Conventions
 *   - Arrays are Fortran column-major; a wavefunction block is (ld x nb)
 *     doubles, grid index x fastest (kinetic_sol_module.f90:85).
 *   - Band/k/spin indices are 1-based as in Fortran.  Only k = 1 (Gamma) is
 *     supported; s selects the spin column of Vloc.
 *   - A wavefunction pointer may be device memory, a host address inside a
 *     range registered with rsdft_gpu_register_wf (then its device mirror is
 *     used and kept current; rsdft_gpu_sync_to_host copies it back), or plain
 *     host memory (copied in and out around the call).
 *   - Small arrays (esp, res, occ, Hsub, Vsub, forces, tables) may be host or
 *     device memory.
 *   - No entry falls back to a CPU implementation.
 *   - Not thread-safe; one CUDA stream per process (rsdft_gpu_set_stream).
 */
#ifndef RSDFT_GPU_H
#define RSDFT_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define RSDFT_OK 0
#define RSDFT_EINVAL (-1)    /* bad argument (size, index, NULL) */
#define RSDFT_ENOTINIT (-2)  /* rsdft_gpu_init / set_grid not called */
#define RSDFT_ECUDA (-3)     /* CUDA / cuBLAS error */
#define RSDFT_ESOLVER (-4)   /* cuSOLVER failure or info != 0 (e.g. overlap not SPD) */
#define RSDFT_ENOMEM (-5)    /* device allocation failed */
#define RSDFT_EUNSUP (-6)    /* unsupported option (k != 1, Md > 8, ...) */
#define RSDFT_ETIMEOUT (-7)  /* a kernel's bounded wait ran out (reported at the next sync) */
#define RSDFT_ECHECK (-8)    /* debug build: an in-kernel index check failed (reported at the next sync) */

/* precision modes of the eigensolver entries; the name gives the operand
 * split of the tensor-core contractions (CG sweeps run in FP32 in every
 * mixed mode; Cholesky, the subspace eigensolve and the closing residuals
 * stay FP64) */
#define RSDFT_MODE_FP64 0          /* plain all-FP64 form */
#define RSDFT_MODE_MIXED_BF16X3 1  /* 3-term split-BF16 (6 products, 24 significant bits) */
#define RSDFT_MODE_MIXED_TF32 2    /* 2-term split-TF32, kind::tf32 (3 products, ~22 bits: FP32 accuracy) */
#define RSDFT_MODE_MIXED_BF16X2 3  /* 2-term split-BF16 (3 products, 16 bits) */

/* ---------------------------------------------------------------- set-up */

/* Bind the library to a CUDA device.  (replaces the MPI/OpenMP start-up the
 * reference does in main.f90:34-60; one rank per GPU) */
int rsdft_gpu_init(int device);
int rsdft_gpu_finalize(void);
const char *rsdft_gpu_last_error(void);
/* Launch on this cudaStream_t from now on (NULL: the library's own stream). */
int rsdft_gpu_set_stream(void *stream);
/* Wait for the stream; reports RSDFT_ETIMEOUT if a kernel aborted on a
 * bounded wait since the last check, RSDFT_ECHECK if (debug build) an
 * in-kernel index check failed. */
int rsdft_gpu_synchronize(void);
/* Number of this library's own kernels launched since it was loaded
 * (diagnostics; library calls such as cuBLAS are not counted).  (no
 * reference counterpart; the reference's timers are watch_module.f90) */
long long rsdft_gpu_kernel_launches(void);
/* Bytes of device workspace the library holds (its named, grow-only
 * buffers; registered wavefunction mirrors and set-up tables not counted).
 * (diagnostics; no reference counterpart) */
long long rsdft_gpu_workspace_bytes(void);
/* Failure-path self test: launch one kernel whose mbarrier wait can never
 * complete, bounded by `cycles` SM clock cycles (1 .. 2^34), after which it
 * sets the error flag exactly as a library kernel whose wait ran out does;
 * the next rsdft_gpu_synchronize returns RSDFT_ETIMEOUT, later calls work.
 * (no reference counterpart: the reference stops the program on errors) */
int rsdft_gpu_selftest_timeout(long long cycles);
/* 1 if this library is the debug build (compiled with RSDFT_GPU_CHECK): the
 * kernels that index memory through stored tables (nonlocal projection,
 * scatter and force gathers) check every such index against its array and,
 * where one is out of range, skip that access and record the check's site,
 * the index and a count in the error word; the next rsdft_gpu_synchronize
 * returns RSDFT_ECHECK and clears it.  0 for the normal build, whose kernels
 * carry no checks.  (the role of the reference's -C bounds-checked build,
 * make.inc.org:62,76) */
int rsdft_gpu_checked_build(void);
/* Debug-build self test: launch one kernel whose check of an index one past
 * the end of an n-element device buffer fails (the access is skipped);
 * the next rsdft_gpu_synchronize returns RSDFT_ECHECK, later calls work.
 * RSDFT_EUNSUP in the normal build, which launches nothing. */
int rsdft_gpu_selftest_check(void);

/* Grid and FD kinetic coefficients: Ngrid(1:3), Md, coef_lap0, coef_lap(3,Md)
 * (axis-major: coef_lap[axis*Md + m-1]), Hgrid(1:3), ggg(1:3), dV.
 * (replaces init_kinetic, kinetic_module.f90:20-153, and the module state of
 * kinetic_variables.f90 / rgrid_module read by op_kinetic_sol) */
int rsdft_gpu_set_grid(const int *ngrid, int md, double coef_lap0, const double *coef_lap,
                       const double *hgrid, const double *ggg, double dv);

/* Local potential Vloc(ML, nspin).  (replaces Vloc of localpot_module.f90:18-25) */
int rsdft_gpu_set_vloc(const double *vloc, long ml, int nspin);

/* Nonlocal KB tables in projector-major CSR (0-based): lma_ptr[nzlma+1],
 * jjp[nnz] (grid index, ascending per projector), uv[nnz], iuv[nzlma] (+-1),
 * amap[nzlma] (0-based atom), duvdr[nnz*3] (d uV / d R_atom, may be NULL).
 * (replaces uVk, JJP, MJJ, iuV, amap of ps_nloc2_variables.f90:3-28 filled by
 * prep_ps_nloc2 / prep_uvk_ps_nloc2, ps_nloc2_module.f90:56-1190, and the
 * duVdR table of calc_force_ps_nloc2 :1489-1586) */
int rsdft_gpu_set_nonlocal(int nzlma, const int *lma_ptr, const int *jjp, const double *uv,
                           const int *iuv, const int *amap, int natom, const double *duvdr);

/* Device mirror of a host wavefunction array unk(ML, MB) (copied in now).
 * (replaces the residency of wf_module's unk(ML_0:ML_1, MB, MK, MS),
 * wf_module.f90:118) */
int rsdft_gpu_register_wf(double *unk, long ml, int mb);
int rsdft_gpu_unregister_wf(double *unk);
int rsdft_gpu_sync_to_host(double *unk);
int rsdft_gpu_sync_to_device(double *unk);

/* ----------------------------------------------------------- hot path */

/* htpsi(n1:n2, ib1:ib2) = H tpsi: FD kinetic + Vloc + nonlocal KB.
 * (replaces hamiltonian(k,s,tpsi,htpsi,n1,n2,ib1,ib2),
 * hamiltonian_module.f90:20-72) */
int rsdft_gpu_hamiltonian(int k, int s, const double *tpsi, double *htpsi, int n1, int n2, int ib1,
                          int ib2);

/* The three operators of hamiltonian, apart, for a caller that splits the
 * grid over ranks (each rank's context holds its slab extended by halo
 * planes, and the projector entries of its own points):
 *   op_local:            htpsi = (T + Vloc(:, s)) tpsi on the z planes
 *                        [z0, z0 + nz) of the context's grid (other planes
 *                        of htpsi untouched), kinetic and local potential
 *                        only (replaces op_kinetic + op_localpot,
 *                        hamiltonian_module.f90:42,50).  The stencil wraps
 *                        periodically in z over the context's n3 planes, so
 *                        on a slab extended by Md halo planes either side
 *                        (z0 = Md, nz = n3 - 2 Md) it reads no wrapped plane;
 *   op_nonlocal_project: uvunk(lma, b) = iuV dV sum_j uV(j, lma) tpsi(JJP(j), b)
 *                        over the context's projector entries, uvunk
 *                        (nzlma, nb) column-major (ps_nloc2_op_module.f90:
 *                        161-175: a rank's partial sums, which the ranks add
 *                        up as :179-250 do);
 *   op_nonlocal_add:     htpsi(JJP(j), b) += uV(j, lma) uvunk(lma, b)
 *                        (ps_nloc2_op_module.f90:255-263).
 * tpsi/htpsi as for rsdft_gpu_hamiltonian (ld >= ML); uvunk host or device. */
int rsdft_gpu_op_local(int s, const double *tpsi, double *htpsi, long ld, int nb, int z0, int nz);
int rsdft_gpu_op_nonlocal_project(const double *tpsi, long ld, int nb, double *uvunk);
int rsdft_gpu_op_nonlocal_add(const double *uvunk, double *htpsi, long ld, int nb);

/* Capacity, in doubles (4 MiB), of the static scratch of
 * rsdft_gpu_hamiltonian_noalloc. */
#define RSDFT_NOALLOC_SCRATCH_VALUES 524288L

/* The same H psi as rsdft_gpu_hamiltonian, for callers that cannot allocate
 * device memory while they run: a host code that has handed all of its GPU
 * memory to its own pool, or that must not wait on the allocator's implicit
 * device synchronisation inside a latency-bound loop.  No counterpart in the
 * reference.
 *  - It calls no cudaMalloc/cudaFree and no allocating library routine.  Its
 *    only scratch, the projection coefficients (nb x nzlma values), sits in a
 *    static device array of RSDFT_NOALLOC_SCRATCH_VALUES doubles that every
 *    GPU loading this library holds until exit.  A call with
 *    (ib2-ib1+1) * nzlma above that returns RSDFT_EINVAL; split the bands.
 *  - tpsi and htpsi must be device memory or lie in a registered
 *    wavefunction: nothing is staged.
 *  - rsdft_gpu_init looks up the array's device address for its device.  The
 *    first launch of a kernel can still make the CUDA driver load that
 *    kernel's code (lazy module loading), which the driver allocates: make
 *    one call at set-up, before the caller's own pool takes the memory and
 *    before any stream capture.
 *  - All calls share the one array: calls that overlap on the GPU (other
 *    streams, other host threads) race.  Each call overwrites every value it
 *    reads, so no clearing is needed between calls. */
int rsdft_gpu_hamiltonian_noalloc(int k, int s, const double *tpsi, double *htpsi, int n1, int n2,
                                  int ib1, int ib2);

/* Band-by-band preconditioned CG, all bands advanced concurrently (exact:
 * SWGS = 0 keeps bands independent).  ncg line steps, mloop preconditioner
 * sweeps, ipc = 4 (hprsdft preconditioner) or 0 (none); mode per above.
 * (replaces conjugate_gradient(n1,n2,MB,k,s,unk,esp,res), cg_module.f90:54-94
 * -> conjugate_gradient_1 :97-430, preconditioning cgpc_module.f90:126-155 ->
 * precond_hprsdft cgpc_hprsdft_module.f90:126-263) */
int rsdft_gpu_conjugate_gradient(int n1, int n2, int mb, int k, int s, double *unk, double *esp,
                                 double *res, int ncg, int mloop, int ipc, int mode);

/* Orthonormalise unk(:, n0:n1) in the dV metric; the result is the unique Q
 * of the QR factorisation with positive diag(R), the output of the recursive
 * blocked Gram-Schmidt.  nblk/nblk1 are accepted for interface parity.
 * (replaces gram_schmidt(n0,n1,k,s) -> gram_schmidt_t,
 * gram_schmidt_module.f90:28-56, gram_schmidt_t_module.f90:84-316) */
int rsdft_gpu_gram_schmidt(int n0, int n1, int k, int s, double *unk, long ld, int nblk, int nblk1,
                           int mode);

/* Hsub = dV * psi^T (H psi), lower triangle (upper set to zero), MB x MB with
 * leading dimension ldh.  (replaces subspace_mate_sl(k,s),
 * subspace_mate_sl_module.f90:27-366, on a 1x1 process grid) */
int rsdft_gpu_subspace_mate(int k, int s, const double *unk, long ld, int mb, double *hsub, int ldh);

/* Eigen-decomposition of the symmetric Hsub (lower triangle read): esp(MB)
 * ascending, Vsub(MB, MB) eigenvectors.  (replaces subspace_solv_sl(k,s),
 * subspace_solv_sl_module.f90:15-134, pdsyevd on a 1x1 grid) */
int rsdft_gpu_subspace_solv(int mb, const double *hsub, int ldh, double *esp, double *vsub, int ldv);

/* unk <- unk * Vsub.  (replaces subspace_rotv_sl(k,s),
 * subspace_rotv_sl_module.f90:24-135) */
int rsdft_gpu_subspace_rotv(int k, int s, double *unk, long ld, int mb, const double *vsub, int ldv);

/* Pieces of gram_schmidt_t / subspace_diag_la for a caller that splits the
 * grid over ranks: each rank forms its partial sums over its own points, the
 * ranks add them up (mpi_allreduce over comm_grid), and every rank solves the
 * small problem redundantly and rotates its own rows.
 *   gram:             C(m, n) = alpha a^T b over `rows` rows (leading
 *                     dimension ld; sym = 1 returns the symmetric part of a
 *                     square product), on the FP64 tensor pipe (replaces the
 *                     dgemm before gram_schmidt_t_module.f90:194 and the
 *                     dsyr2k of subspace_diag_la_module.f90:96);
 *   overlap_cholesky: S = R^T R, rinv = R^-1 (upper, lower triangle zero),
 *                     kappa = (max diag R / min diag R)^2, the conditioning
 *                     gate of the one-pass step (the normalisations of
 *                     gram_schmidt_t_module.f90:84-316 in triangular form);
 *   rr_reduced:       R^-T Hsub R^-1 = V diag(esp) V^T, w = R^-1 V (Hsub's
 *                     upper triangle read), the eigenproblem after
 *                     subspace_diag_la_module.f90:122 and the rotation
 *                     matrix of :200 composed with the Gram-Schmidt one.
 * Matrices host or device, column-major. */
int rsdft_gpu_gram(const double *a, const double *b, long ld, long rows, int m, int n, double alpha, int sym,
                   double *c, int ldc);
int rsdft_gpu_overlap_cholesky(int mb, const double *s, int lds, double *rinv, int ldr, double *kappa);
int rsdft_gpu_rr_reduced(int mb, const double *rinv, int ldr, const double *hsub, int ldh, double *esp,
                         double *w, int ldw);
/* unk(1:rows, 1:mb) <- unk * v for device (or registered) unk with leading
 * dimension ld: the rotation of subspace_rotv_sl_module.f90:92 on a rank's
 * own rows. */
int rsdft_gpu_rotate(double *unk, long ld, long rows, int mb, const double *v, int ldv);

/* Rayleigh-Ritz in span(unk): Hsub = dV/2 (psi^T H psi + (H psi)^T psi),
 * eigen-decomposition, rotation; esp(MB) out.  (replaces subspace_diag(k,s)
 * -> subspace_diag_la, subspace_diag_module.f90:17-25,
 * subspace_diag_la_module.f90:18-232) */
int rsdft_gpu_subspace_diag(int k, int s, double *unk, long ld, int mb, double *esp, int mode);

/* gram_schmidt followed by subspace_diag, as calc_sweep calls them
 * (sweep_module.f90:152-155), in one Rayleigh-Ritz step: overlap Cholesky
 * S = R^T R, eigen-decomposition of R^-T Hsub R^-1 and one rotation by
 * R^-1 V.  Same eigenvalues and orthonormal bands as the pair (replaces
 * gram_schmidt_t_module.f90:84-316 + subspace_diag_la_module.f90:18-232);
 * an ill-conditioned overlap takes the explicit CholeskyQR2 + subspace_diag
 * path. */
int rsdft_gpu_orth_subspace_diag(int k, int s, double *unk, long ld, int mb, double *esp, int mode);

/* One sweep iteration for (k, s) as calc_sweep runs it (sweep_module.f90:
 * 150-155): conjugate_gradient, then gram_schmidt + subspace_diag as in
 * rsdft_gpu_orth_subspace_diag.  esp(MB) receives the Ritz values, res(MB)
 * the CG residuals; ld must equal ML.  In the mixed modes the FP32 bands of
 * the CG sweep feed the Rayleigh-Ritz step directly (FP32 H psi, exact BF16
 * split) and the rotated bands are written back in FP64. */
int rsdft_gpu_eigensolver_sweep(int k, int s, double *unk, long ld, int mb, double *esp, double *res, int ncg,
                                int mloop, int ipc, int mode);

/* calc_sweep's loop for the Gamma point with the bands kept on the device:
 * for iter = 1..diter, for every spin s = 1..nspin, the sweep of
 * rsdft_gpu_eigensolver_sweep on unk(:, :, s) (spin s at unk + (s-1) ld mb),
 * then esp_gather (nothing to gather on one process), calc_fermi
 * (Methfessel-Paxton order kinteg, smearing ekbt, nelectron electrons; fixed
 * spin moment dspn while iter <= nfixed when nspin = 2) and conv_check:
 * iconv_check 2 or 3 stops once max |esp - esp0| over bands 1..mb_ref of
 * every spin is below tol_esp (3 also returns res = |esp - esp0|, -1 below
 * tol_esp; 2 returns the CG residuals).  esp (mb, nspin) holds esp0 of the
 * first iteration on entry and the Ritz values on exit; occ (mb, nspin) the
 * occupations; *iter_out the iteration the loop stopped at, *conv_out 1 if
 * it converged; *efermi (may be NULL) the Fermi level.  iconv_check 1 (the
 * total-energy test) needs the SCF total energy: RSDFT_EUNSUP.
 * (replaces calc_sweep, sweep_module.f90:60-226, with esp_gather,
 * esp_gather_module.f90:11-61, calc_fermi, fermi_mp_module.f90:95-284, and
 * conv_check, sweep_module.f90:228-280) */
int rsdft_gpu_calc_sweep(double *unk, long ld, int mb, int nspin, double *esp, double *res, double *occ,
                         int diter, int iconv_check, double tol_esp, int mb_ref, double nelectron, int nfixed,
                         double dspn, double ekbt, int kinteg, int ncg, int mloop, int ipc, int mode,
                         int *iter_out, int *conv_out, double *efermi);

/* e(ns:ne) = dV <wf_n|H wf_n>, FP64 (no normalisation, as the reference).
 * (replaces esp_calc(k,s,wf,n1,n2,ns,ne,e), esp_calc_module.f90:15-49) */
int rsdft_gpu_esp_calc(int k, int s, const double *wf, int n1, int n2, int ns, int ne, double *e);

/* FP64 Rayleigh quotients and residual norms of nb bands: e(n) = dV <wf|H wf>,
 * res(n) = dV |H wf - e(n) wf|^2 (the quantity cg_module.f90:213 reports as
 * res, times 4 / c1^2 = 1).  The final FP64 pass of the mixed forms.  (no
 * single reference routine: esp_calc_module.f90:15-49 plus the residual of
 * cg_module.f90:186-213) */
int rsdft_gpu_residual(int k, int s, const double *wf, long ld, int nb, double *e, double *res);

/* Norm-conserving nonlocal force force2(3, MI) (column-major, i.e. xyz of
 * atom 1 first) for bands with occ(n) != 0.  (replaces
 * calc_force_ps_nloc2(MI,force2), ps_nloc2_module.f90:1281-1811) */
int rsdft_gpu_force_nloc(int mi, const double *unk, long ld, int mb, const double *occ,
                         double *force2);

/* Adjoint (vector-Jacobian product) of hpsi with respect to the local
 * potential and the atom positions.  For y = H psi and cotangent chi:
 *   dL_dv[r]    += sum_n chi_n(r) psi_n(r)                     (ML)
 *   dL_dr[3a+k] += sum_n sum_{lma in a} iuV dV [ (chi.d_k uV)(uV.psi)
 *                                              + (chi.uV)(d_k uV.psi) ]
 * If chi == NULL, chi_n = occ[n] * dV * psi_n, which makes the outputs the
 * gradients of E = sum_n occ_n <psi_n|H|psi_n> dV (then -dL_dr is the
 * Hellmann-Feynman nonlocal force).  The outputs are overwritten.
 * (no single reference routine: differentiates op_localpot,
 * localpot_module.f90:27-81, and op_ps_nloc2_hp, ps_nloc2_op_module.f90:136-270;
 * the position part is the contraction of calc_force_ps_nloc2,
 * ps_nloc2_module.f90:1601-1773) */
int rsdft_gpu_hpsi_adjoint(const double *psi, const double *chi, long ld, int nb, const double *occ,
                           double *dl_dv, double *dl_dr);

/* Electron density of one (k, spin) block: rho(r) = sum_n occ(n) unk(r,n)^2
 * over the mb bands (occ(n) = 0 skipped), rho(ML) overwritten; a caller with
 * several k points or spins adds the blocks.  (replaces the NCPP branch of
 * calc_density, density_module.f90:115-138, for one block; no symmetry
 * operations) */
int rsdft_gpu_calc_density(const double *unk, long ld, int mb, const double *occ, double *rho);

/* ------------------------------------------------------ wavefunction file */

/* Write unk(ML, mb, mk, ms) (band stride ld, k stride ld*mb, spin stride
 * ld*mb*mk; real Gamma data) to the wavefunction file of RSDFT, record for
 * record: Fortran sequential unformatted records with 4-byte length markers;
 * header, LL2(3,ML) grid map (x fastest), occ(mb,mk,ms), aa(3,3), bb(3,3),
 * kbb(3,mmbz), the single-process layout records, then one record per band
 * n = mbwr1..mbwr2 for every k and spin.  oc = 4 or 5 stores the bands in
 * FP32, oc >= 10 writes the old format (no lattice or layout records), any
 * other oc FP64.  io_ctrl = 0 puts everything in path; io_ctrl = 3 puts the
 * band records in path.00000.  mbwr1/mbwr2 outside 1..mb are replaced by
 * 1 and mb as the reference does.  occ, aa, bb and kbb may be NULL (zeros).
 * unk may be a plain host array, a registered one (its device mirror is
 * written) or device memory (both copied band by band through pinned
 * buffers while the previous band is written).
 * (replaces simple_wf_io_write(file_wf,IO_ctrl,OC,SYStype=0,MBwr1,MBwr2),
 * io_write_module.f90:19-264, for one process) */
int rsdft_gpu_write_wf(const char *path, const double *unk, long ld, int mb, int mk, int ms, int mbwr1, int mbwr2,
                       int oc, int io_ctrl, const int *ngrid, const double *occ, const double *aa,
                       const double *bb, int mmbz, const double *kbb);

/* Read a wavefunction file written by RSDFT (new or old format, FP64 or
 * FP32 bands, io_ctrl 0 or 3 as for the writer) into unk(ML, mb, mk, ms):
 * the grid must match ngrid; grid points are placed through the file's
 * LL2 map; bands, k points and spins beyond mb, mk, ms are skipped.
 * occ(mb,mk,ms), if not NULL, receives the file's occupations over the
 * common ranges.  info[13], if not NULL, receives the header: ML, ML1, ML2,
 * ML3, MB, MB1, MB2, MK, MS, MMBZ, IO_ctrl, OC, TYPE_WF (the old format has
 * no MK..TYPE_WF: mk, ms, 0, 0, 0, 0 are reported).  unk as for the writer:
 * a registered array's device mirror, or device memory, is filled band by
 * band through pinned buffers.
 * (replaces simple_wf_io_read(file_wf,SYStype=0,IO_ctrl,...),
 * io_read_module.f90:15-521, for one process) */
int rsdft_gpu_read_wf(const char *path, double *unk, long ld, int mb, int mk, int ms, int io_ctrl,
                      const int *ngrid, double *occ, int *info);

/* ------------------------------------------ density and potential file */

/* Write the density/potential file of RSDFT (vrho.dat1) record for record:
 * the version record, ML and ngrid, LL2(3,ML) (x fastest), the lattice
 * aa(3,3), Nelement and Natom, aa_atom(3,natom), ki_atom(natom),
 * zn_atom(nelement), efermi, then for each spin s rho(:,s), vloc(:,s), vh
 * (s = 1 only) and vxc(:,s).  rho, vloc and vxc are (ML, nspin) arrays, vh
 * is (ML); each may be a host array, a registered one (its device mirror is
 * written) or device memory.
 * (replaces the density/potential branch of write_data, io_module.f90:97-226,
 * for one process) */
int rsdft_gpu_write_vrho(const char *path, const int *ngrid, const double *aa, int nelement, int natom,
                         const double *aa_atom, const int *ki_atom, const int *zn_atom, double efermi, int nspin,
                         const double *rho, const double *vloc, const double *vh, const double *vxc);

/* Read a density/potential file written by RSDFT (with or without the
 * version record) into rho, vloc, vxc (ML, nspin) and vh (ML), each a host
 * array, a registered one or device memory, or NULL to skip it; the grid must
 * match ngrid and the values are placed through the file's LL2 map.
 * *efermi (if not NULL) receives the Fermi energy of a versioned file and is
 * left untouched for an unversioned one, as in the reference.
 * (replaces the VRHO branch of read_data, io_module.f90:283-432, for one
 * process) */
int rsdft_gpu_read_vrho(const char *path, const int *ngrid, int nspin, double *rho, double *vloc, double *vh,
                        double *vxc, double *efermi);

#ifdef __cplusplus
}
#endif

#endif /* RSDFT_GPU_H */
