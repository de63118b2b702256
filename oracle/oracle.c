/*
 * Oracle: CPU restatement of RSDFT's Kohn-Sham eigensolver inner loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker and the timed
 * CPU baseline; the product (rsdft_b200/ and its CUDA library) never links,
 * loads or calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it.
 *
 * Every routine restates one reference routine of j-iwata/RSDFT v1.3.0
 * (paths relative to its src/ directory), real Gamma-point build
 * (-D_DRSDFT_), one MPI rank, keeping the reference's loop order and
 * per-point summation order:
 *
 *   oracle_hamiltonian   hamiltonian_module.f90:20-72
 *     kinetic            kinetic_sol_module.f90:72-77 (diagonal), :129-149
 *                        (Gamma, orthorhombic stencil), periodic halo as
 *                        built by bc_module.f90:464-474 / bcset_3
 *     local potential    localpot_module.f90:68-74
 *     nonlocal           ps_nloc2_op_module.f90:161-175 (uVunk), :255-263
 *                        (scatter-add)
 *   oracle_dot           ext0/dotp.f90:1-27
 *   oracle_precond       cgpc_hprsdft_module.f90:126-263 + precond_cg_mat2_omp
 *                        :281-348 (IPC = 4)
 *   oracle_dsygv2        LAPACK dsygv(itype=1,'V','U',n=2) as called at
 *                        cg_module.f90:318: dpotrf, dsygst, dsyev (dlaev2
 *                        rotation for the 2x2 tridiagonal), back-transform
 *   oracle_cg            conjugate_gradient_1, cg_module.f90:97-430 (band by
 *                        band, MB_d = 1, cggs no-op since SWGS = 0)
 *   oracle_force_nloc    calc_force_ps_nloc2 band loop and accumulation,
 *                        ps_nloc2_module.f90:1601-1654, :1760-1773
 *
 * Dot products use a fixed blocked order (blocks of 1024, then the block sums
 * in order) so results do not depend on the thread count.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXMD 16

static struct {
    int n1, n2, n3, md;
    long ML;
    double c0;              /* coef_lap0 + const_k2 (Gamma: const_k2 = 0) */
    double cl[3][MAXMD];    /* coef_lap(axis, m) */
    double dV;
    const double *vloc;     /* Vloc(ML) for the spin in use */
    int nzlma;
    const int *lma_ptr;     /* CSR offsets per projector */
    const int *jjp;         /* 0-based grid index, sorted per projector */
    const double *uv;
    const int *iuv;
    double pc_c, pc_c1, pc_c2, pc_c3; /* preconditioner operator */
} H;

int oracle_set_hamiltonian(int n1, int n2, int n3, int md, double coef_lap0,
                           const double *coef_lap /* [3][md], axis major */, double dV,
                           const double *vloc, int nzlma, const int *lma_ptr,
                           const int *jjp, const double *uv, const int *iuv,
                           double pc_c, double pc_c1, double pc_c2, double pc_c3)
{
    if (md < 1 || md > MAXMD) return -1;
    H.n1 = n1; H.n2 = n2; H.n3 = n3; H.md = md;
    H.ML = (long)n1 * n2 * n3;
    H.c0 = coef_lap0;
    for (int a = 0; a < 3; ++a)
        for (int m = 0; m < md; ++m) H.cl[a][m] = coef_lap[a * md + m];
    H.dV = dV;
    H.vloc = vloc;
    H.nzlma = nzlma; H.lma_ptr = lma_ptr; H.jjp = jjp; H.uv = uv; H.iuv = iuv;
    H.pc_c = pc_c; H.pc_c1 = pc_c1; H.pc_c2 = pc_c2; H.pc_c3 = pc_c3;
    return 0;
}

static inline int wrap(int i, int n) { i %= n; return i < 0 ? i + n : i; }

/* kinetic + local for one band (kinetic_sol_module.f90:72-77,129-149;
 * localpot_module.f90:73).  The per-point order is the reference's: the
 * diagonal term first, then for m = 1..Md the x, y, z pairs, then Vloc. */
static void kin_loc_band(const double *t, double *h)
{
    const int n1 = H.n1, n2 = H.n2, n3 = H.n3, md = H.md;
#pragma omp parallel for schedule(static)
    for (int i3 = 0; i3 < n3; ++i3) {
        for (int i2 = 0; i2 < n2; ++i2) {
            for (int i1 = 0; i1 < n1; ++i1) {
                long j = i1 + (long)n1 * (i2 + (long)n2 * i3);
                double v = H.c0 * t[j];
                for (int m = 1; m <= md; ++m) {
                    long xm = wrap(i1 - m, n1) + (long)n1 * (i2 + (long)n2 * i3);
                    long xp = wrap(i1 + m, n1) + (long)n1 * (i2 + (long)n2 * i3);
                    long ym = i1 + (long)n1 * (wrap(i2 - m, n2) + (long)n2 * i3);
                    long yp = i1 + (long)n1 * (wrap(i2 + m, n2) + (long)n2 * i3);
                    long zm = i1 + (long)n1 * (i2 + (long)n2 * wrap(i3 - m, n3));
                    long zp = i1 + (long)n1 * (i2 + (long)n2 * wrap(i3 + m, n3));
                    v = v + H.cl[0][m - 1] * (t[xm] + t[xp])
                          + H.cl[1][m - 1] * (t[ym] + t[yp])
                          + H.cl[2][m - 1] * (t[zm] + t[zp]);
                }
                h[j] = v + H.vloc[j] * t[j];
            }
        }
    }
}

/* ps_nloc2_op_module.f90:161-175 for one band: uVunk(lma) = iuV*dV*sum uV*psi */
static void nloc_project_band(const double *t, double *uvunk)
{
    for (int lma = 0; lma < H.nzlma; ++lma) {
        double s = 0.0;
        for (int j = H.lma_ptr[lma]; j < H.lma_ptr[lma + 1]; ++j) s = s + H.uv[j] * t[H.jjp[j]];
        uvunk[lma] = H.iuv[lma] * H.dV * s;
    }
}

/* ps_nloc2_op_module.f90:255-263: htpsi(JJP) += uV * uVunk(lma) */
static void nloc_scatter_band(const double *uvunk, double *h)
{
    for (int lma = 0; lma < H.nzlma; ++lma)
        for (int j = H.lma_ptr[lma]; j < H.lma_ptr[lma + 1]; ++j) h[H.jjp[j]] = h[H.jjp[j]] + H.uv[j] * uvunk[lma];
}

/* hamiltonian(k,s,tpsi,htpsi,n1,n2,ib1,ib2) for nb columns of leading dimension ld.
 * uvunk_out (optional, nzlma x nb column-major) receives the projections. */
int oracle_hamiltonian(const double *tpsi, double *htpsi, long ld, int nb, double *uvunk_out)
{
    double *uvunk = (double *)malloc(sizeof(double) * (H.nzlma > 0 ? H.nzlma : 1));
    for (int b = 0; b < nb; ++b) {
        const double *t = tpsi + (long)b * ld;
        double *h = htpsi + (long)b * ld;
        kin_loc_band(t, h);
        if (H.nzlma > 0) {
            nloc_project_band(t, uvunk);
            nloc_scatter_band(uvunk, h);
            if (uvunk_out) memcpy(uvunk_out + (long)b * H.nzlma, uvunk, sizeof(double) * H.nzlma);
        }
    }
    free(uvunk);
    return 0;
}

/* blocked sum of a[i]*b[i], fixed order independent of threads */
static double bsum(const double *a, const double *b, long n)
{
    const long BS = 1024;
    long nblk = (n + BS - 1) / BS;
    double *part = (double *)malloc(sizeof(double) * (nblk > 0 ? nblk : 1));
#pragma omp parallel for schedule(static)
    for (long k = 0; k < nblk; ++k) {
        long s = k * BS, e = s + BS < n ? s + BS : n;
        double acc = 0.0;
        for (long i = s; i < e; ++i) acc += a[i] * b[i];
        part[k] = acc;
    }
    double tot = 0.0;
    for (long k = 0; k < nblk; ++k) tot += part[k];
    free(part);
    return tot;
}

/* dot_product(a,b,c,alpha,n,1): c = alpha * sum a*b (ext0/dotp.f90) */
double oracle_dot(const double *a, const double *b, long n, double alpha)
{
    return bsum(a, b, n) * alpha;
}

/* precond_cg_mat2_omp (cgpc_hprsdft_module.f90:281-348), E0 = 0:
 * f = (c - E0) g + c1 (g[i1+1]+g[i1-1]) + c2 (...) + c3 (...) */
static void precond_mat(const double *g, double *f, double E0)
{
    const int n1 = H.n1, n2 = H.n2, n3 = H.n3;
    const double d = H.pc_c - E0;
#pragma omp parallel for schedule(static)
    for (int i3 = 0; i3 < n3; ++i3)
        for (int i2 = 0; i2 < n2; ++i2)
            for (int i1 = 0; i1 < n1; ++i1) {
                long j = i1 + (long)n1 * (i2 + (long)n2 * i3);
                double v = d * g[j];
                v = v + H.pc_c1 * (g[wrap(i1 + 1, n1) + (long)n1 * (i2 + (long)n2 * i3)] +
                                   g[wrap(i1 - 1, n1) + (long)n1 * (i2 + (long)n2 * i3)])
                      + H.pc_c2 * (g[i1 + (long)n1 * (wrap(i2 + 1, n2) + (long)n2 * i3)] +
                                   g[i1 + (long)n1 * (wrap(i2 - 1, n2) + (long)n2 * i3)])
                      + H.pc_c3 * (g[i1 + (long)n1 * (i2 + (long)n2 * wrap(i3 + 1, n3))] +
                                   g[i1 + (long)n1 * (i2 + (long)n2 * wrap(i3 - 1, n3))]);
                f[j] = v;
            }
}

/* precond_hprsdft for one band (cgpc_hprsdft_module.f90:126-263).
 * On entry Pgk = gk (the caller copies, cg_module.f90:205-209). */
void oracle_precond(const double *gk, double *Pgk, int mloop, double *work /* 3*ML */)
{
    const long ML = H.ML;
    double *rk = work, *pk = work + ML, *ft = work + 2 * ML;
    const double ep = 1e-24;
    if (mloop <= 0) return;
    precond_mat(gk, ft, 0.0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < ML; ++i) { rk[i] = gk[i] - ft[i]; pk[i] = rk[i]; }
    double rr1 = bsum(rk, rk, ML);
    if (rr1 < ep) return;
    for (int iloop = 1; iloop <= mloop; ++iloop) {
        precond_mat(pk, ft, 0.0);
        double pAp = bsum(pk, ft, ML);
        double rr0 = rr1;
        double a = rr0 / pAp;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < ML; ++i) Pgk[i] = Pgk[i] + a * pk[i];
        if (iloop == mloop) break;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < ML; ++i) rk[i] = rk[i] - a * ft[i];
        rr1 = bsum(rk, rk, ML);
        double b = rr1 / rr0;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < ML; ++i) pk[i] = rk[i] + b * pk[i];
    }
}

/* LAPACK dlaev2: eigen-decomposition of [[a,b],[b,c]]; rt1 has the larger
 * absolute value, (cs1, sn1) is its unit eigenvector. */
static void dlaev2_(double a, double b, double c, double *rt1, double *rt2, double *cs1, double *sn1)
{
    double sm = a + c, df = a - c, adf = fabs(df), tb = b + b, ab = fabs(tb);
    double acmx, acmn, rt, cs, ct, tn;
    int sgn1, sgn2;
    if (fabs(a) > fabs(c)) { acmx = a; acmn = c; } else { acmx = c; acmn = a; }
    if (adf > ab) rt = adf * sqrt(1.0 + (ab / adf) * (ab / adf));
    else if (adf < ab) rt = ab * sqrt(1.0 + (adf / ab) * (adf / ab));
    else rt = ab * sqrt(2.0);
    if (sm < 0.0) { *rt1 = 0.5 * (sm - rt); sgn1 = -1; *rt2 = (acmx / *rt1) * acmn - (b / *rt1) * b; }
    else if (sm > 0.0) { *rt1 = 0.5 * (sm + rt); sgn1 = 1; *rt2 = (acmx / *rt1) * acmn - (b / *rt1) * b; }
    else { *rt1 = 0.5 * rt; *rt2 = -0.5 * rt; sgn1 = 1; }
    if (df >= 0.0) { cs = df + rt; sgn2 = 1; } else { cs = df - rt; sgn2 = -1; }
    if (fabs(cs) > ab) { ct = -tb / cs; *sn1 = 1.0 / sqrt(1.0 + ct * ct); *cs1 = ct * *sn1; }
    else {
        if (ab == 0.0) { *cs1 = 1.0; *sn1 = 0.0; }
        else { tn = -cs / tb; *cs1 = 1.0 / sqrt(1.0 + tn * tn); *sn1 = tn * *cs1; }
    }
    if (sgn1 == sgn2) { tn = *cs1; *cs1 = -*sn1; *sn1 = tn; }
}

/* dsygv(1,'V','U',2,A,2,B,2,W,...) for symmetric A, SPD B (column-major 2x2).
 * On return A holds the B-orthonormal eigenvectors (columns) in ascending
 * order of W.  Returns info (0, or >0 if B is not positive definite). */
int oracle_dsygv2(double *A, double *B, double *W)
{
    double a11 = A[0], a12 = A[2], a22 = A[3];
    double b11 = B[0], b12 = B[2], b22 = B[3];
    /* dpotrf('U'): B = U^T U */
    if (!(b11 > 0.0)) return 3;
    double u11 = sqrt(b11);
    double u12 = b12 / u11;
    double t = b22 - u12 * u12;
    if (!(t > 0.0)) return 4;
    double u22 = sqrt(t);
    /* dsygst(1,'U'): C = U^-T A U^-1 */
    double c11 = a11 / (u11 * u11);
    double r12 = a12 / u11;
    double c12 = (r12 - c11 * u12) / u22;
    double c22 = (a22 - 2.0 * u12 * r12 + u12 * u12 * c11) / (u22 * u22);
    /* dsyev on [[c11,c12],[c12,c22]] */
    double rt1, rt2, cs, sn;
    dlaev2_(c11, c12, c22, &rt1, &rt2, &cs, &sn);
    double z1[2], z2[2], w1, w2;
    if (rt1 <= rt2) { w1 = rt1; w2 = rt2; z1[0] = cs; z1[1] = sn; z2[0] = -sn; z2[1] = cs; }
    else { w1 = rt2; w2 = rt1; z1[0] = -sn; z1[1] = cs; z2[0] = cs; z2[1] = sn; }
    W[0] = w1; W[1] = w2;
    /* back-transform x = U^-1 z (dtrsm 'L','U','N') */
    double x12 = z1[1] / u22, x11 = (z1[0] - u12 * x12) / u11;
    double x22 = z2[1] / u22, x21 = (z2[0] - u12 * x22) / u11;
    A[0] = x11; A[1] = x12; A[2] = x21; A[3] = x22;
    return 0;
}

/* conjugate_gradient_1 (cg_module.f90:97-430), real, MB_d = 1, SWGS = 0.
 * unk(ML, MB) column-major, updated in place; esp(MB), res(MB) out.
 * stats (optional, 2 ints): number of hpsi and preconditioner calls. */
int oracle_cg(double *unk, long ML, int MB, double *esp, double *res, int Mcg, int mloop, int *stats)
{
    const double ep0 = 0.0, ep1 = 1e-15, c1 = 2.0;
    const double dV = H.dV;
    if (ML != H.ML) return -1;
    double *hxk = (double *)malloc(sizeof(double) * ML * 8);
    double *hpk = hxk + ML, *gk = hxk + 2 * ML, *Pgk = hxk + 3 * ML, *pk = hxk + 4 * ML, *work = hxk + 5 * ML;
    int nh = 0, npc = 0;
    for (int n = 0; n < MB; ++n) { res[n] = 0.0; esp[n] = 0.0; }
    for (int ns = 0; ns < MB; ++ns) {
        double *x = unk + (long)ns * ML;
        double E1 = 1e10, E, rb, gkgk = 0.0;
        oracle_hamiltonian(x, hxk, ML, 1, NULL); ++nh;
        E = oracle_dot(x, hxk, ML, dV);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < ML; ++i) gk[i] = -c1 * (hxk[i] - E * x[i]);
        rb = oracle_dot(gk, gk, ML, dV);
        for (int icg = 1; icg <= Mcg + 1; ++icg) {
            memcpy(Pgk, gk, sizeof(double) * ML);
            res[ns] = rb / (c1 * c1);
            if (rb < ep0) break;
            if (fabs(E - E1) < ep1) break;
            if (icg == Mcg + 1) break;
            oracle_precond(gk, Pgk, mloop, work); ++npc;
            rb = oracle_dot(Pgk, gk, ML, dV);
            if (icg == 1) memcpy(pk, Pgk, sizeof(double) * ML);
            else {
                double bk = rb / gkgk;
#pragma omp parallel for schedule(static)
                for (long i = 0; i < ML; ++i) pk[i] = Pgk[i] + bk * pk[i];
            }
            gkgk = rb;
            oracle_hamiltonian(pk, hpk, ML, 1, NULL); ++nh;
            double v[6];
            v[0] = oracle_dot(x, x, ML, dV);
            v[1] = oracle_dot(pk, x, ML, dV);
            v[2] = oracle_dot(pk, pk, ML, dV);
            v[3] = oracle_dot(x, hxk, ML, dV);
            v[4] = oracle_dot(pk, hxk, ML, dV);
            v[5] = oracle_dot(pk, hpk, ML, dV);
            double bt[4] = {v[0], v[1], v[1], v[2]};
            double ut[4] = {v[3], v[4], v[4], v[5]};
            double W[2];
            int info = oracle_dsygv2(ut, bt, W);
            if (info != 0) { free(hxk); return 100 + info; }
            if (fabs(W[0] - E) > 1e-1 && fabs(W[1] - E) <= 1e-1) {
                ut[0] = ut[2]; ut[1] = ut[3]; W[0] = W[1];
            }
            if (ut[0] < 0.0) { ut[0] = -ut[0]; ut[1] = -ut[1]; }
            E1 = E;
            E = W[0];
            const double u11 = ut[0], u21 = ut[1], w = W[0];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < ML; ++i) hxk[i] = u11 * hxk[i] + u21 * hpk[i];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < ML; ++i) gk[i] = -c1 * (hxk[i] - w * (u11 * x[i] + u21 * pk[i]));
            rb = oracle_dot(gk, gk, ML, dV);
            if (rb / res[ns] > 1e8) { E = E1; continue; }
#pragma omp parallel for schedule(static)
            for (long i = 0; i < ML; ++i) x[i] = u11 * x[i] + u21 * pk[i];
        }
        esp[ns] = E;
    }
    if (stats) { stats[0] = nh; stats[1] = npc; }
    free(hxk);
    return 0;
}

/* Nonlocal force (calc_force_ps_nloc2 band loop, ps_nloc2_module.f90:1601-1654,
 * accumulation :1760-1773): for each band with occ != 0,
 *   w0(lma) = iuV * (-2 occ dV^2) * sum_j uV(j) psi(JJP(j))
 *   w_k(lma) = sum_j duVdR(k, j) psi(JJP(j))
 *   force2(k, amap(lma)) += w0 * w_k
 * duv is (nnz, 3) row-major: the derivative of uV with respect to the atom
 * position.  force2 is (natom, 3) row-major, zeroed here. */
int oracle_force_nloc(const double *unk, long ML, int MB, const double *occ, const double *duv,
                      const int *amap, int natom, double *force2)
{
    (void)ML;
    for (long i = 0; i < 3L * natom; ++i) force2[i] = 0.0;
    for (int n = 0; n < MB; ++n) {
        if (occ[n] == 0.0) continue;
        const double *psi = unk + (long)n * H.ML;
        const double c = -2.0 * occ[n] * H.dV * H.dV;
        for (int lma = 0; lma < H.nzlma; ++lma) {
            double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
            for (int j = H.lma_ptr[lma]; j < H.lma_ptr[lma + 1]; ++j) w0 = w0 + H.uv[j] * psi[H.jjp[j]];
            w0 = H.iuv[lma] * c * w0;
            for (int j = H.lma_ptr[lma]; j < H.lma_ptr[lma + 1]; ++j) {
                double p = psi[H.jjp[j]];
                w1 = w1 + duv[3L * j + 0] * p;
                w2 = w2 + duv[3L * j + 1] * p;
                w3 = w3 + duv[3L * j + 2] * p;
            }
            int a = amap[lma];
            force2[3 * a + 0] += w0 * w1;
            force2[3 * a + 1] += w0 * w2;
            force2[3 * a + 2] += w0 * w3;
        }
    }
    return 0;
}

/* ===========================================================================
 * Reference path of the nonlocal force's derivative table (test
 * infrastructure): the tabulated, interpolated duVdR of calc_force_ps_nloc2
 * (ps_nloc2_module.f90:1489-1586), from the radial derivative tables of
 * ps_nloc2_init_derivative (ps_nloc2_init_module.f90:219-301), polint /
 * dpolint (polint_module.f90:11-77) and Ylm / Plm (ylm_module.f90:10-122).
 * The product path uses the analytic derivative instead; these routines let
 * the tests measure how far the two are apart.
 * =========================================================================== */

/* Plm (ylm_module.f90:75-122): associated Legendre function with the
 * Condon-Shortley phase, upward recurrence in l */
static double ref_plm(int L, int M, double xi)
{
    double x = xi;
    if (fabs(fabs(x) - 1.0) < 1e-13) x = x < 0.0 ? -1.0 : 1.0;
    double pmm = 1.0;
    if (M > 0) {
        const double somx2 = sqrt((1.0 - x) * (1.0 + x));
        double fact = 1.0;
        for (int i = 1; i <= M; ++i) {
            pmm = -pmm * fact * somx2;
            fact += 2.0;
        }
    }
    if (L == M) return pmm;
    double pmmp1 = x * (2.0 * M + 1.0) * pmm;
    if (L == M + 1) return pmmp1;
    double pll = 0.0;
    for (int ll = M + 2; ll <= L; ++ll) {
        pll = (x * (2.0 * ll - 1.0) * pmmp1 - (ll + M - 1.0) * pmm) / (ll - M);
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}

/* Ylm(x,y,z,L,M) (ylm_module.f90:10-72): real spherical harmonics */
double oracle_ylm(double x, double y, double z, int L, int Min)
{
    const double pi = 3.141592653589793238, pi4 = 4.0 * pi;
    const int M = Min < 0 ? -Min : Min;
    if (L == 0) return 1.0 / sqrt(pi4);
    if (x == 0.0 && y == 0.0 && z == 0.0) return 0.0;
    double c = 1.0;
    for (int k = L - M + 1; k <= L + M; ++k) c *= (double)k;
    const double Clm = sqrt((2.0 * L + 1.0) / (c * pi4));
    const double r = sqrt(x * x + y * y + z * z), ct = z / r;
    double phi;
    if (fabs(x) < 1e-10) phi = 0.5 * pi * (y < 0.0 ? -1.0 : 1.0);
    else {
        phi = atan(y / x);
        if (x < 0) phi += pi;
    }
    if (Min > 0) return sqrt(2.0) * Clm * ref_plm(L, M, ct) * cos(phi * M);
    if (Min == 0) return Clm * ref_plm(L, M, ct);
    if (M % 2 == 0) return -sqrt(2.0) * Clm * ref_plm(L, M, ct) * sin(phi * M);
    return sqrt(2.0) * Clm * ref_plm(L, M, ct) * sin(phi * M);
}

/* polint (polint_module.f90:11-41): Neville interpolation of ya(xa) at x; dy
 * is the change of the averaged last column, the error estimate */
static void ref_polint(const double *xa, const double *ya, int n, double x, double *y, double *dy, double *f0)
{
    for (int i = 0; i < n; ++i) f0[i] = ya[i];
    double f0nm = ya[0], f0nm_0 = f0nm;
    for (int m = 1; m <= n - 1; ++m) {
        for (int i = 0; i < n - m; ++i) {
            const double a = x - xa[i], b = x - xa[i + m];
            f0[i] = (b * f0[i] - a * f0[i + 1]) / (b - a);
        }
        f0nm_0 = f0nm;
        double s = 0.0;
        for (int i = 0; i < n - m; ++i) s += f0[i];
        f0nm = s / (n - m);
    }
    *y = f0[0];
    *dy = f0nm - f0nm_0;
}

/* dpolint (polint_module.f90:44-77): the derivative of the Neville
 * polynomial at x, with the same kind of error estimate */
static void ref_dpolint(const double *xa, const double *ya, int n, double x, double *y, double *dy, double *f0,
                        double *f1)
{
    for (int i = 0; i < n; ++i) {
        f0[i] = ya[i];
        f1[i] = 0.0;
    }
    double f1nm = (ya[1] - ya[0]) / (xa[1] - xa[0]), f1nm_0 = f1nm;
    for (int m = 1; m <= n - 1; ++m) {
        for (int i = 0; i < n - m; ++i) {
            const double a = x - xa[i], b = x - xa[i + m];
            f1[i] = (f0[i] - f0[i + 1] + b * f1[i] - a * f1[i + 1]) / (b - a);
            f0[i] = (b * f0[i] - a * f0[i + 1]) / (b - a);
        }
        f1nm_0 = f1nm;
        double s = 0.0;
        for (int i = 0; i < n - m; ++i) s += f1[i];
        f1nm = s / (n - m);
    }
    *y = f1[0];
    *dy = f1nm - f1nm_0;
}

/* ps_nloc2_init_derivative (ps_nloc2_init_module.f90:219-301) for one
 * orbital of angular momentum L with radial function viod on rad[0..nrc-1]:
 * dv(i) = the dpolint derivative over the windows [i-m, i+m] (m = 1..20,
 * clipped) with the smallest error estimate, then for J = |L-1| .. L+1
 * (row t = J - |L-1| of out, nrc values each)
 *   out = sqrt(4 pi / 3) (rad^2 dv + (2 + L(L+1) - J(J+1))/2 rad viod) */
int oracle_dviod(const double *rad, const double *viod, int nrc, int L, double *out)
{
    double *dv = malloc(sizeof(double) * (size_t)nrc), *f0 = malloc(sizeof(double) * 64),
           *f1 = malloc(sizeof(double) * 64);
    if (!dv || !f0 || !f1) { free(dv); free(f0); free(f1); return -1; }
    for (int i = 0; i < nrc; ++i) {
        double y0 = 0.0, dy0 = 1e10, y, dy;
        for (int m = 1; m <= 20; ++m) {
            const int m1 = i - m > 0 ? i - m : 0, m2 = i + m < nrc - 1 ? i + m : nrc - 1;
            ref_dpolint(rad + m1, viod + m1, m2 - m1 + 1, rad[i], &y, &dy, f0, f1);
            if (fabs(dy) < dy0) { y0 = y; dy0 = fabs(dy); }
        }
        dv[i] = y0;
    }
    const double c43 = sqrt(4.0 * acos(-1.0) / 3.0);
    const int J0 = L > 0 ? L - 1 : 1 - L;
    for (int J = J0, t = 0; J <= L + 1; ++J, ++t) {
        const double cj = 0.5 * (2.0 + L * (L + 1) - J * (J + 1));
        for (int i = 0; i < nrc; ++i) out[(long)t * nrc + i] = c43 * (rad[i] * rad[i] * dv[i] + cj * rad[i] * viod[i]);
    }
    free(dv); free(f0); free(f1);
    return 0;
}

/* duVdR(1:3, j, lma) of calc_force_ps_nloc2 (ps_nloc2_module.f90:1507-1586,
 * the polint branch) for the npt points of one projector (L, m):
 * d[3 j .. 3 j + 2] = point - atom; dviod = oracle_dviod's rows for this
 * orbital; gaunt = the three coupling tables of this (L, m), indexed
 * [k][L1][L1z + L + 1] for L1 = 0 .. L + 1 (k = x, y, z);
 * out[3 j + k] the derivative of uV with respect to the atom position. */
int oracle_duvdr_ref(int L, const double *d, int npt, const double *rad, int nrc, const double *dviod,
                     const double *gaunt, double *out)
{
    const double ep = 1e-8;
    const int J0 = L > 0 ? L - 1 : 1 - L, W = 2 * L + 3, NL1 = L + 2;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (int j = 0; j < npt; ++j) {
        double f0[64];
        const double x = d[3L * j], y = d[3L * j + 1], z = d[3L * j + 2];
        const double r = sqrt(x * x + y * y + z * z);
        double yy1 = 0.0, yy2 = 0.0, yy3 = 0.0;
        for (int L1 = J0; L1 <= L + 1; ++L1) {
            if (!(fabs(x) > 1e-14 || fabs(y) > 1e-14 || fabs(z) > 1e-14 || L1 == 0)) continue;
            const double *dvi = dviod + (long)(L1 - J0) * nrc;
            /* bisection on rad (1-based indices as the reference) */
            int ir0 = 1, ir1 = nrc;
            while (ir1 - ir0 > 1) {
                const int ir = (ir0 + ir1) / 2;
                if (rad[ir - 1] > r) ir1 = ir;
                else ir0 = ir;
            }
            const int ir = ir0;
            double tmp0 = 0.0;
            if (ir <= 2) {
                tmp0 = dvi[1] / (rad[1] * rad[1]);
                if (ir < 1) ++bad;
            } else if (ir <= nrc) {
                double err0 = 1e10, tmp1, err;
                for (int im = 1; im <= 20; ++im) {
                    const int m1 = ir - im > 1 ? ir - im : 1, m2 = ir + im < nrc ? ir + im : nrc;
                    ref_polint(rad + m1 - 1, dvi + m1 - 1, m2 - m1 + 1, r, &tmp1, &err, f0);
                    if (fabs(err) < err0) {
                        tmp0 = tmp1;
                        err0 = fabs(err);
                        if (err0 < ep) break;
                    }
                }
                tmp0 = tmp0 / (r * r);
            }
            for (int L1z = -L1; L1z <= L1; ++L1z) {
                const double t1 = tmp0 * oracle_ylm(x, y, z, L1, L1z);
                const long g = (long)L1 * W + (L1z + L + 1);
                yy1 += t1 * gaunt[0L * NL1 * W + g];
                yy2 += t1 * gaunt[1L * NL1 * W + g];
                yy3 -= t1 * gaunt[2L * NL1 * W + g];
            }
        }
        out[3L * j] = yy1;
        out[3L * j + 1] = yy2;
        out[3L * j + 2] = yy3;
    }
    return bad ? -1 : 0;
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
