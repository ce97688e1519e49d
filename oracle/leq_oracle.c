/*
 * leq_oracle.c -- TEST INFRASTRUCTURE ONLY (see leq_oracle.h).
 *
 * Plain-C restatement of the reference's FP64 LEQ_BICGS path for a serial,
 * non-cyclic, non-cut-cell MFIX box.  It is the parity checker for the CUDA
 * library and, compiled with OpenMP, the timed CPU baseline.  The OpenMP
 * regions sit where the reference has them (model/leq_bicgs.f:211,285,303,335,
 * 365,432; model/leqsol_mod.f:188-189,216-217,497,510); the dot products stay
 * serial, as DOT_PRODUCT_PAR is in a serial run (model/leqsol_mod.f:1125-1136).
 *
 * Build with -ffp-contract=off so that every product and sum rounds the way a
 * non-FMA Fortran build of the reference rounds it.
 */
#include "leq_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define DIAG(a, g, d) ((a) + (int64_t)((d) + 3) * (g)->n)

static inline int64_t cell(const orc_geom *g, int i, int j, int k)
{
    /* FUNIJK for a serial run: ijk = j + c0 + i*c1 + k*c2 with c0 = -c1 - c2 + 0 (0-based here) */
    return (int64_t)(j - 1) + (int64_t)(i - 1) * g->jmax2 + (int64_t)(k - 1) * g->jmax2 * g->imax2;
}

/* Neighbour increments of a serial box (model/set_increments.f:73-113): clamped at
 * the array edge (IM1(I) = MAX(ISTART3, I-1)), or, along a cyclic axis, wrapping
 * the interior cells 2..m-1 (IP1(I) = IMAP_C(IMAP_C(I)+1), with IMAP_C(IMAX2) =
 * IMIN1 and IMAP_C(IMIN2) = IMAX1, model/dmp_modules/gridmap_mod.f:496-503).  t is
 * 1-based, m the extent including the wall layer; the result is in cells of
 * that axis. */
static inline int64_t inc_m(int t, int m, int cyc)
{
    if (cyc && t >= 2 && t <= m - 1) return t == 2 ? (int64_t)(m - 3) : -1;
    return t > 1 ? -1 : 0;
}
static inline int64_t inc_p(int t, int m, int cyc)
{
    if (cyc && t >= 2 && t <= m - 1) return t == m - 1 ? -(int64_t)(m - 3) : 1;
    return t < m ? 1 : 0;
}
#define CYC_X(g) (((g)->cyclic & 1) != 0)
#define CYC_Y(g) (((g)->cyclic & 2) != 0)
#define CYC_Z(g) (((g)->cyclic & 4) != 0)

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ random stream */
/* splitmix64 output function (Steele, Lea & Flood, OOPSLA 2014), used counter-wise so
 * that every cell's draw is independent of evaluation order.  Replaces Fortran
 * RANDOM_NUMBER in model/leq_bicgs.f:298. */
static inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double orc_uniform(uint64_t seed, uint64_t tag, uint64_t idx)
{
    uint64_t key = mix64(seed * 0x9E3779B97F4A7C15ULL + tag * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL);
    uint64_t v = mix64(key + (idx + 1) * 0x9E3779B97F4A7C15ULL);
    return (double)(v >> 11) * 0x1.0p-53;
}

/* ------------------------------------------------------------------ LEQ_MATVEC */
/* model/leqsol_mod.f:166-254 (non-reindexed branch).  The core-cell loop and the
 * boundary loop evaluate the same expression; only the neighbour offsets differ,
 * and for a serial box they are the clamped ones of model/set_increments.f:80-109. */
void orc_matvec(const orc_geom *g, const double *a, const double *x, double *y)
{
    const int64_t c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
    const int imax2 = g->imax2, jmax2 = g->jmax2, kmax2 = g->kmax2, do_k = g->do_k;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= kmax2; ++k) {
        for (int i = 1; i <= imax2; ++i) {
            const int64_t im = inc_m(i, imax2, CYC_X(g)) * c1, ip = inc_p(i, imax2, CYC_X(g)) * c1;
            const int64_t km = do_k ? inc_m(k, kmax2, CYC_Z(g)) * c2 : 0, kp = do_k ? inc_p(k, kmax2, CYC_Z(g)) * c2 : 0;
            const int64_t base = cell(g, i, 1, k);
            for (int j = 1; j <= jmax2; ++j) {
                const int64_t p = base + (j - 1);
                const int64_t jm = inc_m(j, jmax2, CYC_Y(g)), jp = inc_p(j, jmax2, CYC_Y(g));
                double s = am2[p] * x[p + jm] + am1[p] * x[p + im] + a0[p] * x[p] + ap1[p] * x[p + ip] +
                           ap2[p] * x[p + jp];
                if (do_k) {
                    s = s + am3[p] * x[p + km];
                    s = s + ap3[p] * x[p + kp];
                }
                y[p] = s;
            }
        }
    }
}

/* ------------------------------------------------------------------ DOT_PRODUCT_PAR */
/* Serial run: the Fortran DOT_PRODUCT intrinsic over the whole array,
 * model/leqsol_mod.f:1125-1127, accumulated in index order. */
double orc_dot(const double *x, const double *y, int64_t n)
{
    double s = 0.0;
    for (int64_t p = 0; p < n; ++p) s = s + x[p] * y[p];
    return s;
}

/* ------------------------------------------------------------------ DGTSV */
/* Gaussian elimination with partial pivoting on a tridiagonal, NRHS = 1:
 * model/DGTSV.f:92-163 (factor) and :231-246 (back solve).  Zero-based arrays:
 * dl[0..n-2], d[0..n-1], du[0..n-2], b[0..n-1].  Returns INFO. */
int orc_dgtsv(int n, double *dl, double *d, double *du, double *b)
{
    if (n < 0) return -1;
    if (n == 0) return 0;
    double fact, temp;
    for (int i = 0; i < n - 2; ++i) {
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                fact = dl[i] / d[i];
                d[i + 1] = d[i + 1] - fact * du[i];
                b[i + 1] = b[i + 1] - fact * b[i];
            } else {
                return i + 1;
            }
            dl[i] = 0.0;
        } else {
            fact = d[i] / dl[i];
            d[i] = dl[i];
            temp = d[i + 1];
            d[i + 1] = du[i] - fact * temp;
            dl[i] = du[i + 1];
            du[i + 1] = -fact * dl[i];
            du[i] = temp;
            temp = b[i];
            b[i] = b[i + 1];
            b[i + 1] = temp - fact * b[i + 1];
        }
    }
    if (n > 1) {
        const int i = n - 2;
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                fact = dl[i] / d[i];
                d[i + 1] = d[i + 1] - fact * du[i];
                b[i + 1] = b[i + 1] - fact * b[i];
            } else {
                return i + 1;
            }
        } else {
            fact = d[i] / dl[i];
            d[i] = dl[i];
            temp = d[i + 1];
            d[i + 1] = du[i] - fact * temp;
            du[i] = temp;
            temp = b[i];
            b[i] = b[i + 1];
            b[i + 1] = temp - fact * b[i + 1];
        }
    }
    if (d[n - 1] == 0.0) return n;
    b[n - 1] = b[n - 1] / d[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
    return 0;
}

/* ------------------------------------------------------------------ line sweeps */
/* LEQ_IKSWEEP, model/leqsol_mod.f:851-921: one J-line at (I,K).  On INFO != 0 the
 * line is left as it was (:910-914). */
int orc_iksweep(const orc_geom *g, int i, int k, double *var, const double *a, const double *b)
{
    const int L = g->jmax2;
    const int64_t c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    const int64_t im = inc_m(i, g->imax2, CYC_X(g)) * c1, ip = inc_p(i, g->imax2, CYC_X(g)) * c1;
    const int64_t km = inc_m(k, g->kmax2, CYC_Z(g)) * c2, kp = inc_p(k, g->kmax2, CYC_Z(g)) * c2;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)(L + 1));
    double *cc = buf, *dd = buf + (L + 1), *ee = buf + 2 * (L + 1), *bb = buf + 3 * (L + 1);
    const int64_t base = cell(g, i, 1, k);
    for (int j = 0; j < L; ++j) {
        const int64_t p = base + j;
        dd[j] = a0[p];
        cc[j] = am2[p];
        ee[j] = ap2[p];
        bb[j] = b[p] - am1[p] * var[p + im] - ap1[p] * var[p + ip] - am3[p] * var[p + km] - ap3[p] * var[p + kp];
    }
    cc[0] = 0.0;
    ee[L - 1] = 0.0;
    const int info = orc_dgtsv(L, cc + 1, dd, ee, bb);
    if (info == 0)
        for (int j = 0; j < L; ++j) var[base + j] = bb[j];
    free(buf);
    return info;
}

/* LEQ_ISWEEP, model/leqsol_mod.f:767-834: the 2-D J-line at I (K = 1). */
int orc_isweep(const orc_geom *g, int i, double *var, const double *a, const double *b)
{
    const int L = g->jmax2;
    const int64_t c1 = g->jmax2;
    const int64_t im = inc_m(i, g->imax2, CYC_X(g)) * c1, ip = inc_p(i, g->imax2, CYC_X(g)) * c1;
    const double *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2);
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)(L + 1));
    double *cc = buf, *dd = buf + (L + 1), *ee = buf + 2 * (L + 1), *bb = buf + 3 * (L + 1);
    const int64_t base = cell(g, i, 1, 1);
    for (int j = 0; j < L; ++j) {
        const int64_t p = base + j;
        dd[j] = a0[p];
        cc[j] = am2[p];
        ee[j] = ap2[p];
        bb[j] = b[p] - am1[p] * var[p + im] - ap1[p] * var[p + ip];
    }
    cc[0] = 0.0;
    ee[L - 1] = 0.0;
    const int info = orc_dgtsv(L, cc + 1, dd, ee, bb);
    if (info == 0)
        for (int j = 0; j < L; ++j) var[base + j] = bb[j];
    free(buf);
    return info;
}

/* LEQ_JKSWEEP, model/leqsol_mod.f:939-1004: the I-line at (J,K). */
int orc_jksweep(const orc_geom *g, int j, int k, double *var, const double *a, const double *b)
{
    const int L = g->imax2;
    const int64_t c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    const int64_t jm = inc_m(j, g->jmax2, CYC_Y(g)), jp = inc_p(j, g->jmax2, CYC_Y(g));
    const int64_t km = inc_m(k, g->kmax2, CYC_Z(g)) * c2, kp = inc_p(k, g->kmax2, CYC_Z(g)) * c2;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)(L + 1));
    double *cc = buf, *dd = buf + (L + 1), *ee = buf + 2 * (L + 1), *bb = buf + 3 * (L + 1);
    for (int i = 0; i < L; ++i) {
        const int64_t p = cell(g, i + 1, j, k);
        dd[i] = a0[p];
        cc[i] = am1[p];
        ee[i] = ap1[p];
        bb[i] = b[p] - am2[p] * var[p + jm] - ap2[p] * var[p + jp] - am3[p] * var[p + km] - ap3[p] * var[p + kp];
    }
    (void)c1;
    cc[0] = 0.0;
    ee[L - 1] = 0.0;
    const int info = orc_dgtsv(L, cc + 1, dd, ee, bb);
    if (info == 0)
        for (int i = 0; i < L; ++i) var[cell(g, i + 1, j, k)] = bb[i];
    free(buf);
    return info;
}

/* LEQ_IJSWEEP, model/leqsol_mod.f:1021-1086: the K-line at (I,J). */
int orc_ijsweep(const orc_geom *g, int i, int j, double *var, const double *a, const double *b)
{
    const int L = g->kmax2;
    const int64_t c1 = g->jmax2;
    const int64_t jm = inc_m(j, g->jmax2, CYC_Y(g)), jp = inc_p(j, g->jmax2, CYC_Y(g));
    const int64_t im = inc_m(i, g->imax2, CYC_X(g)) * c1, ip = inc_p(i, g->imax2, CYC_X(g)) * c1;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)(L + 1));
    double *cc = buf, *dd = buf + (L + 1), *ee = buf + 2 * (L + 1), *bb = buf + 3 * (L + 1);
    for (int k = 0; k < L; ++k) {
        const int64_t p = cell(g, i, j, k + 1);
        dd[k] = a0[p];
        cc[k] = am3[p];
        ee[k] = ap3[p];
        bb[k] = b[p] - am2[p] * var[p + jm] - ap2[p] * var[p + jp] - am1[p] * var[p + im] - ap1[p] * var[p + ip];
    }
    cc[0] = 0.0;
    ee[L - 1] = 0.0;
    const int info = orc_dgtsv(L, cc + 1, dd, ee, bb);
    if (info == 0)
        for (int k = 0; k < L; ++k) var[cell(g, i, j, k + 1)] = bb[k];
    free(buf);
    return info;
}

/* ------------------------------------------------------------------ LEQ_MSOLVE */
/* model/leqsol_mod.f:286-598: Var = B (SETGUESS, :342-357), then one action per
 * character of the four-character sweep string.  Returns 0, or -12 when DGTSV
 * fails inside a JK/IJ sweep (the reference aborts there, :991-996, :1073-1078). */
int orc_msolve(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep,
               int *skips)
{
    const int64_t n = g->n;
    int nskip = 0;
    memcpy(var, b, sizeof(double) * (size_t)n);
    for (int it = 0; it < 4; ++it) {
        const char ch = sweep[it];
        const int do_i = (ch == 'I' || ch == 'i');
        const int do_kk = (ch == 'K' || ch == 'k');
        const int do_all = (ch == 'A' || ch == 'a');
        const int do_rb = (ch == 'R' || ch == 'r');
        if (!g->do_k) {
            /* two-dimensional branch, :372-391 */
            if (do_i)
                for (int i = 1; i <= g->imax2; ++i) nskip += orc_isweep(g, i, var, a, b) != 0;
            if (do_rb) {
                /* an odd number of cyclic interior cells puts the wrapped lines in one
                 * colour: the serial loop order then decides what each one reads */
                const int par_ok = !(CYC_X(g) && ((g->imax2 - 2) & 1));
                int s1 = 0, s2 = 0;
#pragma omp parallel for reduction(+ : s1) schedule(static) if (par_ok)
                for (int i = 1; i <= g->imax2; i += 2) s1 += orc_isweep(g, i, var, a, b) != 0;
#pragma omp parallel for reduction(+ : s2) schedule(static) if (par_ok)
                for (int i = 2; i <= g->imax2; i += 2) s2 += orc_isweep(g, i, var, a, b) != 0;
                nskip += s1 + s2;
            }
            continue;
        }
        if (do_all) {
            /* :398-470, every loop sequential as in the reference */
            const int jsize = g->jmax2, ksize = g->kmax2, isize = g->imax2;
            for (int icase = 1; icase <= 2; ++icase)
                for (int jk = icase; jk <= ksize * jsize; jk += 2) {
                    int k = (jk % jsize != 0) ? jk / jsize + 1 : jk / jsize;
                    int j = (jk - 1 - (k - 1) * jsize) + 1 + (k % 2);
                    if (j > jsize) j = j - jsize;
                    if (orc_jksweep(g, j, k, var, a, b) != 0) return -12;
                }
            for (int icase = 1; icase <= 2; ++icase)
                for (int ij = icase; ij <= jsize * isize; ij += 2) {
                    int j = (ij % isize != 0) ? ij / isize + 1 : ij / isize;
                    int i = (ij - 1 - (j - 1) * isize) + 1 + (j % 2);
                    if (i > isize) i = i - isize;
                    if (orc_ijsweep(g, i, j, var, a, b) != 0) return -12;
                }
            for (int icase = 1; icase <= 2; ++icase)
                for (int ik = icase; ik <= ksize * isize; ik += 2) {
                    int k = (ik % isize != 0) ? ik / isize + 1 : ik / isize;
                    int i = (ik - 1 - (k - 1) * isize) + 1 + (k % 2);
                    if (i > isize) i = i - isize;
                    nskip += orc_iksweep(g, i, k, var, a, b) != 0;
                }
        }
        if (do_rb) {
            /* :497-522: first the lines with (i+k) odd, then (i+k) even */
            /* the I wrap stays inside one k iteration; the K wrap of an odd number of
             * cyclic interior cells joins two k iterations of one colour */
            const int par_ok = !(CYC_Z(g) && ((g->kmax2 - 2) & 1));
            int s1 = 0, s2 = 0;
#pragma omp parallel for reduction(+ : s1) schedule(static) if (par_ok)
            for (int k = 1; k <= g->kmax2; ++k)
                for (int i = (k % 2 != 0) ? 2 : 1; i <= g->imax2; i += 2) s1 += orc_iksweep(g, i, k, var, a, b) != 0;
#pragma omp parallel for reduction(+ : s2) schedule(static) if (par_ok)
            for (int k = 1; k <= g->kmax2; ++k)
                for (int i = (k % 2 != 0) ? 1 : 2; i <= g->imax2; i += 2) s2 += orc_iksweep(g, i, k, var, a, b) != 0;
            nskip += s1 + s2;
        }
        if (do_i) /* :567-574 */
            for (int k = 1; k <= g->kmax2; ++k)
                for (int i = 1; i <= g->imax2; ++i) nskip += orc_iksweep(g, i, k, var, a, b) != 0;
        if (do_kk) /* :575-582 */
            for (int i = 1; i <= g->imax2; ++i)
                for (int k = 1; k <= g->kmax2; ++k) nskip += orc_iksweep(g, i, k, var, a, b) != 0;
    }
    if (skips) *skips += nskip;
    return 0;
}

/* LEQ_MSOLVE1 (DIAG), model/leqsol_mod.f:719-746 */
void orc_msolve1(const orc_geom *g, const double *b, const double *a, double *var)
{
    const double *a0 = DIAG(a, g, 0);
    const int64_t n = g->n;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) var[p] = b[p] / a0[p];
}

/* ------------------------------------------------------------------ unit scaling */
/* model/leq_bicgs.f:194-233: every row divided by max|A(ijk,:)| through a
 * multiplication by its reciprocal; a zero row flags IER = -2. */
int orc_scale(const orc_geom *g, double *a, double *b)
{
    const int64_t n = g->n;
    int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        double m = fabs(a[p]);
        for (int d = 1; d < 7; ++d) {
            const double v = fabs(a[(int64_t)d * n + p]);
            if (isnan(m) || v > m) m = v;
        }
        if (m > 0.0) {
            const double oam = 1.0 / m;
            for (int d = 0; d < 7; ++d) a[(int64_t)d * n + p] = a[(int64_t)d * n + p] * oam;
            b[p] = b[p] * oam;
        } else {
            bad |= 1;
        }
    }
    return bad ? -2 : 0;
}

/* ------------------------------------------------------------------ LEQ_CG0 unit scaling */
/* model/leq_cg.f:197-211: every row multiplied by the reciprocal of its diagonal
 * A(ijk,0), with no zero test (a zero diagonal gives infinities, as in the
 * reference). */
void orc_scale_diag(const orc_geom *g, double *a, double *b)
{
    const int64_t n = g->n;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        const double oam = 1.0 / a[3 * n + p];
        for (int d = 0; d < 7; ++d) a[(int64_t)d * n + p] = a[(int64_t)d * n + p] * oam;
        b[p] = b[p] * oam;
    }
}

/* ------------------------------------------------------------------ LEQ_BICGS0 */
#define SMALL_NUMBER 1.0e-15
#define RATIOTOL ((double)0.2f) /* DOUBLE PRECISION, PARAMETER :: ratiotol = 0.2 (a REAL literal) */

static int pc_mode(const char *pc)
{
    /* model/leq_bicgs.f:74-87: CHARACTER(LEN=4) compared with blank padding */
    if (!memcmp(pc, "LINE", 4)) return 2;
    if (!memcmp(pc, "DIAG", 4)) return 1;
    if (!memcmp(pc, "NONE", 4)) return 0;
    return -1;
}

static int msolve_t(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep, int *skips);

/* transposed: LEQ_BICGS0t (model/leq_bicgst.f:102-627), whose scaling has no zero-row
 * test (:214-229) and whose preconditioner is LEQ_MSOLVEt */
/* icheck: 0, or MINIMIZE_DOTPRODUCTS with the convergence test every icheck
 * iterations (ICHECK_BICGS, model/leq_bicgs.f:372,411,439; LEQ_BICGSt tests every
 * fifth, model/leq_bicgst.f:514): no Snorm exit, Rnorm formed only when tested. */
static int bicgs_run_x(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                       const char *pc, int itmax, uint64_t rt_seed, int max_exec, orc_stats *st, int transposed,
                       int icheck);

static int bicgs_run(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                     const char *pc, int itmax, uint64_t rt_seed, int max_exec, orc_stats *st)
{
    return bicgs_run_x(g, var, a, b, sweep, tol, pc, itmax, rt_seed, max_exec, st, 0, 0);
}

static int bicgs_run_x(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                       const char *pc, int itmax, uint64_t rt_seed, int max_exec, orc_stats *st, int transposed,
                       int icheck)
{
    memset(st, 0, sizeof(*st));
    st->exit_kind = -1;
    const int mode = pc_mode(pc);
    if (mode < 0) {
        st->ier = -10;
        return -10;
    }
    const int64_t n = g->n;
    if (transposed) {
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < g->n; ++p) {
            double m = 0.0;
            for (int q = 0; q < 7; ++q)
                if (fabs(a[q * g->n + p]) > m) m = fabs(a[q * g->n + p]);
            const double oam = 1.0 / m;
            for (int q = 0; q < 7; ++q) a[q * g->n + p] = a[q * g->n + p] * oam;
            b[p] = b[p] * oam;
        }
    } else if (orc_scale(g, a, b) != 0) {
        st->ier = -2;
        st->exit_kind = 4;
        return -2;
    }
    double *work = (double *)calloc((size_t)(8 * n), sizeof(double));
    double *R = work, *Rt = work + n, *P = work + 2 * n, *Pp = work + 3 * n, *S = work + 4 * n,
           *Sp = work + 5 * n, *T = work + 6 * n, *V = work + 7 * n;
    const double tolmin = DBL_EPSILON;

    orc_matvec(g, a, var, R);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) R[p] = b[p] - R[p];
    const double rnorm0 = sqrt(orc_dot(R, R, n));
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) Rt[p] = R[p] + (2.0 * orc_uniform(rt_seed, 0xA1, (uint64_t)p) - 1.0) * 1.0e-6 * rnorm0;

    double rnorm = 0.0, rho_m1 = 0.0, rho_m2 = 0.0, alpha_m1 = 0.0, omega_m1 = 0.0;
    int iter = 1, converged = 0, ier = 0, executed = 0, iter_tot_add = 0;
    int exit_kind = 3;
    for (int i = 1; i <= itmax; ++i) {
        if (max_exec >= 0 && executed >= max_exec) break;
        ++executed;
        rho_m1 = orc_dot(Rt, R, n);
        if (rho_m1 == 0.0) {
            ier = (i != 1) ? -2 : 0;
            st->ier = ier;
            st->iterations = iter;
            st->exit_kind = 2;
            st->rnorm0 = rnorm0;
            st->rnorm = rnorm;
            free(work);
            return ier;
        }
        if (i == 1) {
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) P[p] = R[p];
        } else {
            const double beta = (rho_m1 / rho_m2) * (alpha_m1 / omega_m1);
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) P[p] = R[p] + beta * (P[p] - omega_m1 * V[p]);
        }
        const double *Ph = P;
        if (mode == 2) {
            if ((transposed ? msolve_t(g, P, a, Pp, sweep, &st->line_info_skips)
                            : orc_msolve(g, P, a, Pp, sweep, &st->line_info_skips)) != 0) { ier = -12; break; }
            Ph = Pp;
        } else if (mode == 1) {
            orc_msolve1(g, P, a, Pp);
            Ph = Pp;
        }
        orc_matvec(g, a, Ph, V);
        const double rtv = orc_dot(Rt, V, n);
        const double alpha = rho_m1 / rtv;
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) S[p] = R[p] - alpha * V[p];
        const double snorm = icheck ? 1.0 : sqrt(orc_dot(S, S, n));
        if (!icheck && snorm <= tolmin) {
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) var[p] = var[p] + alpha * Ph[p];
            converged = 1;
            exit_kind = 1;
            break;
        }
        const double *Sh = S;
        if (mode == 2) {
            if ((transposed ? msolve_t(g, S, a, Sp, sweep, &st->line_info_skips)
                            : orc_msolve(g, S, a, Sp, sweep, &st->line_info_skips)) != 0) { ier = -12; break; }
            Sh = Sp;
        } else if (mode == 1) {
            orc_msolve1(g, S, a, Sp);
            Sh = Sp;
        }
        orc_matvec(g, a, Sh, T);
        const double txs = orc_dot(T, S, n);
        double txt = orc_dot(T, T, n);
        if (txt == 0.0) txt = SMALL_NUMBER;
        const double omega = txs / txt;
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            var[p] = var[p] + alpha * Ph[p] + omega * Sh[p];
            R[p] = S[p] - omega * T[p];
        }
        if (!icheck || iter % icheck == 0) {
            rnorm = sqrt(orc_dot(R, R, n));
            if (rnorm <= tol * rnorm0) {
                iter_tot_add = iter + 1;
                converged = 1;
                exit_kind = 0;
                break;
            }
        }
        ++iter;
        rho_m2 = rho_m1;
        alpha_m1 = alpha;
        omega_m1 = omega;
    }
    if (ier == -12) {
        st->ier = -12;
        st->exit_kind = -1;
        free(work);
        return -12;
    }
    /* model/leq_bicgs.f:486-495 */
    if (!converged) converged = ((double)(float)rnorm <= tol * rnorm0);
    ier = 0;
    if (!converged) {
        ier = -1;
        iter_tot_add = iter;
        if ((double)(float)rnorm >= RATIOTOL * (double)(float)rnorm0) ier = -2;
    }
    st->ier = ier;
    st->iterations = iter;
    st->iter_tot_add = iter_tot_add;
    st->exit_kind = exit_kind;
    st->rnorm0 = rnorm0;
    st->rnorm = rnorm;
    free(work);
    return ier;
}

int orc_leq_bicgs(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                  const char *pc, int itmax, uint64_t rt_seed, orc_stats *st)
{
    return bicgs_run(g, var, a, b, sweep, tol, pc, itmax, rt_seed, -1, st);
}

int orc_leq_bicgs_icheck(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                         const char *pc, int itmax, uint64_t rt_seed, int icheck, orc_stats *st)
{
    return bicgs_run_x(g, var, a, b, sweep, tol, pc, itmax, rt_seed, -1, st, 0, icheck);
}

int orc_leq_bicgs_sample(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                         const char *pc, int itmax, uint64_t rt_seed, int max_exec, orc_stats *st)
{
    return bicgs_run(g, var, a, b, sweep, tol, pc, itmax, rt_seed, max_exec, st);
}

/* ------------------------------------------------------------------ truth oracle */
double orc_true_resid(const orc_geom *g, const double *a, const double *b, const double *x)
{
    const int64_t c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
    long double tot = 0.0L;
#pragma omp parallel for collapse(2) reduction(+ : tot) schedule(static)
    for (int k = 1; k <= g->kmax2; ++k)
        for (int i = 1; i <= g->imax2; ++i) {
            const int64_t im = inc_m(i, g->imax2, CYC_X(g)) * c1, ip = inc_p(i, g->imax2, CYC_X(g)) * c1;
            const int64_t km = g->do_k ? inc_m(k, g->kmax2, CYC_Z(g)) * c2 : 0;
            const int64_t kp = g->do_k ? inc_p(k, g->kmax2, CYC_Z(g)) * c2 : 0;
            const int64_t base = cell(g, i, 1, k);
            for (int j = 1; j <= g->jmax2; ++j) {
                const int64_t p = base + j - 1;
                const int64_t jm = inc_m(j, g->jmax2, CYC_Y(g)), jp = inc_p(j, g->jmax2, CYC_Y(g));
                long double s = (long double)am2[p] * x[p + jm] + (long double)am1[p] * x[p + im] +
                                (long double)a0[p] * x[p] + (long double)ap1[p] * x[p + ip] +
                                (long double)ap2[p] * x[p + jp];
                if (g->do_k) s += (long double)am3[p] * x[p + km] + (long double)ap3[p] * x[p + kp];
                const long double r = (long double)b[p] - s;
                tot += r * r;
            }
        }
    return (double)sqrtl(tot);
}

static void true_resid_vec(const orc_geom *g, const double *a, const double *b, const double *x, double *r)
{
    const int64_t c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    const double *am3 = DIAG(a, g, -3), *am2 = DIAG(a, g, -2), *am1 = DIAG(a, g, -1);
    const double *a0 = DIAG(a, g, 0), *ap1 = DIAG(a, g, 1), *ap2 = DIAG(a, g, 2), *ap3 = DIAG(a, g, 3);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= g->kmax2; ++k)
        for (int i = 1; i <= g->imax2; ++i) {
            const int64_t im = inc_m(i, g->imax2, CYC_X(g)) * c1, ip = inc_p(i, g->imax2, CYC_X(g)) * c1;
            const int64_t km = g->do_k ? inc_m(k, g->kmax2, CYC_Z(g)) * c2 : 0;
            const int64_t kp = g->do_k ? inc_p(k, g->kmax2, CYC_Z(g)) * c2 : 0;
            const int64_t base = cell(g, i, 1, k);
            for (int j = 1; j <= g->jmax2; ++j) {
                const int64_t p = base + j - 1;
                const int64_t jm = inc_m(j, g->jmax2, CYC_Y(g)), jp = inc_p(j, g->jmax2, CYC_Y(g));
                long double s = (long double)am2[p] * x[p + jm] + (long double)am1[p] * x[p + im] +
                                (long double)a0[p] * x[p] + (long double)ap1[p] * x[p + ip] +
                                (long double)ap2[p] * x[p + jp];
                if (g->do_k) s += (long double)am3[p] * x[p + km] + (long double)ap3[p] * x[p + kp];
                r[p] = (double)((long double)b[p] - s);
            }
        }
}

/* Plain right-preconditioned BiCGSTAB (LINE, RSRS) on A d = r, stopping when the
 * recursive residual falls by `drop`; used for refinement steps only. */
static void bicgs_inner(const orc_geom *g, const double *a, const double *r0, double *d, double drop, int maxit,
                        uint64_t seed, double *work)
{
    const int64_t n = g->n;
    double *R = work, *Rt = work + n, *P = work + 2 * n, *Pp = work + 3 * n, *S = work + 4 * n,
           *Sp = work + 5 * n, *T = work + 6 * n, *V = work + 7 * n;
    memset(d, 0, sizeof(double) * (size_t)n);
    memcpy(R, r0, sizeof(double) * (size_t)n);
    const double rn0 = sqrt(orc_dot(R, R, n));
    for (int64_t p = 0; p < n; ++p) Rt[p] = R[p] + (2.0 * orc_uniform(seed, 0xA2, (uint64_t)p) - 1.0) * 1e-6 * rn0;
    double rho_m2 = 1, alpha_m1 = 0, omega_m1 = 1;
    for (int i = 1; i <= maxit; ++i) {
        const double rho = orc_dot(Rt, R, n);
        if (rho == 0.0) break;
        if (i == 1)
            memcpy(P, R, sizeof(double) * (size_t)n);
        else {
            const double beta = (rho / rho_m2) * (alpha_m1 / omega_m1);
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) P[p] = R[p] + beta * (P[p] - omega_m1 * V[p]);
        }
        orc_msolve(g, P, a, Pp, "RSRS", NULL);
        orc_matvec(g, a, Pp, V);
        const double alpha = rho / orc_dot(Rt, V, n);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) S[p] = R[p] - alpha * V[p];
        orc_msolve(g, S, a, Sp, "RSRS", NULL);
        orc_matvec(g, a, Sp, T);
        const double txt = orc_dot(T, T, n);
        const double omega = txt == 0.0 ? 0.0 : orc_dot(T, S, n) / txt;
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            d[p] = d[p] + alpha * Pp[p] + omega * Sp[p];
            R[p] = S[p] - omega * T[p];
        }
        if (sqrt(orc_dot(R, R, n)) <= drop * rn0 || omega == 0.0) break;
        rho_m2 = rho;
        alpha_m1 = alpha;
        omega_m1 = omega;
    }
}

int orc_truth_solve(const orc_geom *g, const double *a, const double *b, double *x, double rtol, int max_iter,
                    uint64_t rt_seed, double *final_rel)
{
    return orc_truth_refine(g, a, b, x, orc_true_resid(g, a, b, x), rtol, max_iter, rt_seed, final_rel);
}

int orc_truth_refine(const orc_geom *g, const double *a, const double *b, double *x, double r0, double rtol,
                     int max_iter, uint64_t rt_seed, double *final_rel)
{
    const int64_t n = g->n;
    double *work = (double *)calloc((size_t)(10 * n), sizeof(double));
    double *r = work + 8 * n, *d = work + 9 * n;
    double rel = 1.0;
    int steps = 0;
    if (r0 == 0.0) {
        rel = 0.0;
    } else {
        for (steps = 0; steps < max_iter; ++steps) {
            true_resid_vec(g, a, b, x, r);
            rel = orc_true_resid(g, a, b, x) / r0;
            if (rel <= rtol) break;
            bicgs_inner(g, a, r, d, 1e-6, 400, rt_seed + (uint64_t)steps, work);
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) x[p] += d[p];
        }
        rel = orc_true_resid(g, a, b, x) / r0;
    }
    if (final_rel) *final_rel = rel;
    free(work);
    return rel <= rtol ? steps : -1;
}

/* ------------------------------------------------------------------ LEQ_CG0 */
/* Preconditioned conjugate gradients, METHOD 5 of SOLVE_LIN_EQ
 * (model/solve_lin_eq.f:173-176, model/leq_cg.f:96-455).  PC dispatch :62-76;
 * R = B - A Var and Rnorm0 :236-259; per iteration Z = MSOLVE(R) :274,
 * rho = (R, Z) with the rho == 0 exit :294-303 (IER 0 at i = 1, else -2, no
 * ITER_TOT update), P = Z or Z + beta P :305-334, Q = A P, alpha = rho / (P, Q)
 * :336-354, R -= alpha Q and Var += alpha P :366-367, Rnorm and the
 * convergence test :396-401; IER rules after the loop :443-450 (the ratio test
 * on REAL() values, ratiotol a REAL literal). */
int orc_leq_cg(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
               const char *pc, int itmax, orc_stats *st)
{
    memset(st, 0, sizeof(*st));
    st->exit_kind = -1;
    const int mode = pc_mode(pc);
    if (mode < 0) {
        st->ier = -10;
        return -10;
    }
    const int64_t n = g->n;
    orc_scale_diag(g, a, b);
    double *work = (double *)calloc((size_t)(4 * n), sizeof(double));
    double *R = work, *P = work + n, *Z = work + 2 * n, *Q = work + 3 * n;
    orc_matvec(g, a, var, R);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) R[p] = b[p] - R[p];
    const double rnorm0 = sqrt(orc_dot(R, R, n));

    double rnorm = 0.0, rho_m2 = 0.0;
    int iter = 1, converged = 0, iter_tot_add = 0, exit_kind = 3;
    for (int i = 1; i <= itmax; ++i) {
        const double *Zp = R;
        if (mode == 2) {
            if (orc_msolve(g, R, a, Z, sweep, &st->line_info_skips) != 0) {
                st->ier = -12;
                free(work);
                return -12;
            }
            Zp = Z;
        } else if (mode == 1) {
            orc_msolve1(g, R, a, Z);
            Zp = Z;
        }
        const double rho = orc_dot(R, Zp, n);
        if (rho == 0.0) {
            const int ier = (i != 1) ? -2 : 0;
            st->ier = ier;
            st->iterations = iter;
            st->exit_kind = 2;
            st->rnorm0 = rnorm0;
            st->rnorm = rnorm;
            free(work);
            return ier;
        }
        if (i == 1) {
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) P[p] = Zp[p];
        } else {
            const double beta = rho / rho_m2;
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) P[p] = Zp[p] + beta * P[p];
        }
        orc_matvec(g, a, P, Q);
        const double pxq = orc_dot(P, Q, n);
        const double alpha = rho / pxq;
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            R[p] = R[p] - alpha * Q[p];
            var[p] = var[p] + alpha * P[p];
        }
        rnorm = sqrt(orc_dot(R, R, n));
        if (rnorm <= tol * rnorm0) {
            iter_tot_add = iter + 1;
            converged = 1;
            exit_kind = 0;
            break;
        }
        ++iter;
        rho_m2 = rho;
    }
    int ier = 0;
    if (!converged) {
        ier = -1;
        iter_tot_add = iter;
        if ((double)(float)rnorm >= RATIOTOL * (double)(float)rnorm0) ier = -2;
    }
    st->ier = ier;
    st->iterations = iter;
    st->iter_tot_add = iter_tot_add;
    st->exit_kind = exit_kind;
    st->rnorm0 = rnorm0;
    st->rnorm = rnorm;
    free(work);
    return ier;
}

/* ------------------------------------------------------------------ LEQ_GMRES0 */
/* ROTMAT (model/leq_gmres.f:593-628): the Givens rotation that zeroes b. */
static void rotmat(double a, double b, double *c, double *s)
{
    if (b == 0.0) {
        *c = 1.0;
        *s = 0.0;
    } else if (fabs(b) > fabs(a)) {
        const double t = a / b;
        *s = 1.0 / sqrt(1.0 + t * t);
        *c = t * *s;
    } else {
        const double t = b / a;
        *c = 1.0 / sqrt(1.0 + t * t);
        *s = t * *c;
    }
}

/* Back substitution of H(1:m,1:m) y = SS(1:m) and Var += V(:,1:m) y with the
 * per-cell sum taken over the basis in order (:362-426, :447-507). */
static void gmres_update(int64_t n, int m, const double *H, int ldh, const double *ss, const double *V, double *var)
{
    double *y = (double *)malloc((size_t)(m > 0 ? m : 1) * sizeof(double));
    for (int i = 0; i < m; ++i) y[i] = ss[i];
    for (int i = m - 1; i >= 0; --i) {
        const double yi = y[i] / H[i + (size_t)i * ldh];
        y[i] = yi;
        for (int j = 0; j < i; ++j) y[j] = y[j] - H[j + (size_t)i * ldh] * yi;
    }
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        double d = 0.0;
        for (int k = 0; k < m; ++k) d = d + V[(size_t)k * n + p] * y[k];
        var[p] = var[p] + d;
    }
    free(y);
}

/* GMRES(ITMAX) with one restart cycle (SOLVE_LIN_EQ passes MAX_IT = 1,
 * model/solve_lin_eq.f:86,147-150,161-171), left-preconditioned by LEQ_MSOLVE
 * with the sweep letters; no unit scaling, A and B untouched.  LEQ_GMRES
 * (model/leq_gmres.f:17-76) returns Var = 0 for B = 0.  LEQ_GMRES0 (:94-584):
 * BNRM2 = ||B|| (:209-218); R = MSOLVE(B - A Var), ERROR0 = ||R|| / BNRM2
 * (:220-246); the Arnoldi loop with modified Gram-Schmidt (:296-327), the
 * rotations and the convergence test (:329-360), the update on convergence
 * (:361-426) or after ITMAX steps with the new true residual (:445-540); IER = 1
 * when not converged (:545-549).  The condition checks of :371-411 run only in a
 * debug build of the reference (JDEBUG = 0) and are not restated. */
int orc_leq_gmres(const orc_geom *g, double *var, const double *a, const double *b, const char *sweep, double tol,
                  int itmax, orc_stats *st)
{
    memset(st, 0, sizeof(*st));
    st->exit_kind = -1;
    const int64_t n = g->n;
    double bmax = 0.0;
    for (int64_t p = 0; p < n; ++p) bmax = fabs(b[p]) > bmax ? fabs(b[p]) : bmax;
    if (bmax == 0.0) {
        for (int64_t p = 0; p < n; ++p) var[p] = 0.0;
        st->exit_kind = 2;
        return 0;
    }
    const int M = itmax > 0 ? itmax : 0;
    double *V = (double *)calloc((size_t)(M + 1) * (size_t)n, sizeof(double));
    double *R = (double *)calloc((size_t)n, sizeof(double)), *T = (double *)calloc((size_t)n, sizeof(double));
    double *W = (double *)calloc((size_t)n, sizeof(double));
    const int ldh = M + 1;
    double *H = (double *)calloc((size_t)ldh * (size_t)(M > 0 ? M : 1), sizeof(double));
    double *cs = (double *)calloc((size_t)M + 1, sizeof(double)), *sn = (double *)calloc((size_t)M + 1, sizeof(double));
    double *ss = (double *)calloc((size_t)M + 2, sizeof(double));
    int skips = 0, rc = 0;
    double bnrm2 = sqrt(orc_dot(b, b, n));
    if (bnrm2 == 0.0) bnrm2 = 1.0;
    orc_matvec(g, a, var, R);
    for (int64_t p = 0; p < n; ++p) T[p] = b[p] - R[p];
    if (orc_msolve(g, T, a, R, sweep, &skips) != 0) rc = -12;
    double norm_r = sqrt(orc_dot(R, R, n));
    double error = norm_r / bnrm2;
    const double error0 = error;
    int steps = 0, converged = 0;
    if (rc == 0) {
        /* the single restart cycle recomputes the same R (:256-283) */
        const double inv = 1.0 / norm_r;
        for (int64_t p = 0; p < n; ++p) V[p] = R[p] * inv;
        for (int k = 0; k < M + 2; ++k) ss[k] = 0.0;
        ss[0] = norm_r;
        for (int i = 0; i < M && !converged; ++i) {
            double *vi = V + (size_t)i * n, *vn = V + (size_t)(i + 1) * n;
            double *h = H + (size_t)i * ldh;
            orc_matvec(g, a, vi, T);
            if (orc_msolve(g, T, a, W, sweep, &skips) != 0) {
                rc = -12;
                break;
            }
            for (int k = 0; k <= i; ++k) {
                const double *vk = V + (size_t)k * n;
                h[k] = orc_dot(W, vk, n);
                for (int64_t p = 0; p < n; ++p) W[p] = W[p] - h[k] * vk[p];
            }
            h[i + 1] = sqrt(orc_dot(W, W, n));
            const double invh = 1.0 / h[i + 1];
            for (int64_t p = 0; p < n; ++p) vn[p] = W[p] * invh;
            for (int k = 0; k < i; ++k) {
                const double d = cs[k] * h[k] + sn[k] * h[k + 1];
                h[k + 1] = -sn[k] * h[k] + cs[k] * h[k + 1];
                h[k] = d;
            }
            rotmat(h[i], h[i + 1], &cs[i], &sn[i]);
            const double d = cs[i] * ss[i];
            ss[i + 1] = -sn[i] * ss[i];
            ss[i] = d;
            h[i] = cs[i] * h[i] + sn[i] * h[i + 1];
            h[i + 1] = 0.0;
            error = fabs(ss[i + 1]) / bnrm2;
            steps = i + 1;
            if (error <= tol * error0) {
                gmres_update(n, i + 1, H, ldh, ss, V, var);
                converged = 1;
            }
        }
        if (rc == 0 && !converged) {
            gmres_update(n, M, H, ldh, ss, V, var);
            orc_matvec(g, a, var, R);
            for (int64_t p = 0; p < n; ++p) T[p] = b[p] - R[p];
            if (orc_msolve(g, T, a, R, sweep, &skips) != 0) rc = -12;
            norm_r = sqrt(orc_dot(R, R, n));
            error = norm_r / bnrm2;
        }
    }
    free(V);
    free(R);
    free(T);
    free(W);
    free(H);
    free(cs);
    free(sn);
    free(ss);
    st->line_info_skips = skips;
    if (rc) {
        st->ier = rc;
        return rc;
    }
    st->ier = (error > tol * error0) ? 1 : 0;
    st->iterations = steps;
    st->exit_kind = st->ier ? 3 : 0;
    st->rnorm0 = error0 * bnrm2;
    st->rnorm = error * bnrm2;
    return st->ier;
}

/* ------------------------------------------------------------------ LEQ_SOR */
/* METHOD 1 (model/solve_lin_eq.f:133-135, model/leq_sor.f:17-122).  Each row is
 * multiplied by 1/A(ijk,0) with A(ijk,0) set to one (:75-85).  Every one of the
 * ITMAX passes forms VAR_tmp = VAR + OMEGA (B - sum_nb A_nb VAR_nb - VAR) from the
 * same VAR (OMEGA = 1, :57, :87-113; the neighbour order differs between 3-D and
 * 2-D), and VAR takes VAR_tmp once after the loop (:115-117), so the result is
 * one point-Jacobi step.  ITER_TOT(VNO) is set, not increased, to the loop
 * counter's final value ITMAX + 1 (:119); IER is left alone.  With ITMAX < 1 the
 * reference copies an array it never wrote; here VAR is left unchanged. */
int orc_leq_sor(const orc_geom *g, double *var, double *a, double *b, int itmax, orc_stats *st)
{
    memset(st, 0, sizeof(*st));
    const int64_t n = g->n, c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    for (int64_t p = 0; p < n; ++p) {
        const double oam = 1.0 / a[3 * n + p];
        a[3 * n + p] = 1.0;
        for (int d = 0; d < 7; ++d)
            if (d != 3) a[(int64_t)d * n + p] = a[(int64_t)d * n + p] * oam;
        b[p] = b[p] * oam;
    }
    st->iter_tot_add = (itmax > 0 ? itmax : 0) + 1;
    st->iterations = st->iter_tot_add;
    st->exit_kind = 3;
    if (itmax < 1) return 0;
    double *tmp = (double *)malloc((size_t)n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        const int64_t line = p / g->jmax2;
        const int j = (int)(p - line * g->jmax2), k = (int)(line / g->imax2), i = (int)(line - (int64_t)k * g->imax2);
        const int64_t jm = j > 0 ? -1 : 0, jp = j < g->jmax2 - 1 ? 1 : 0;
        const int64_t im = i > 0 ? -c1 : 0, ip = i < g->imax2 - 1 ? c1 : 0;
        double v;
        if (g->do_k) {
            const int64_t km = k > 0 ? -c2 : 0, kp = k < g->kmax2 - 1 ? c2 : 0;
            v = b[p] - a[2 * n + p] * var[p + im] - a[4 * n + p] * var[p + ip] - a[1 * n + p] * var[p + jm] -
                a[5 * n + p] * var[p + jp] - a[0 * n + p] * var[p + km] - a[6 * n + p] * var[p + kp] - var[p];
        } else {
            v = b[p] - a[1 * n + p] * var[p + jm] - a[5 * n + p] * var[p + jp] - a[2 * n + p] * var[p + im] -
                a[4 * n + p] * var[p + ip] - var[p];
        }
        tmp[p] = var[p] + 1.0 * v;
    }
    memcpy(var, tmp, (size_t)n * sizeof(double));
    free(tmp);
    return 0;
}

/* ------------------------------------------------------------------ pressure-correction assembly */
/* CONV_PP_G (model/conv_pp_g.f:33-182) followed by SOURCE_PP_G
 * (model/source_pp_g.f:18-214), incompressible (COMPRESSIBLE_PP_G is not
 * called), no Cartesian-grid factors, no shear.  CONV_PP_G writes each face
 * coefficient from the cell below the face (ROP_GE(IJK)*AYZ(IJK) is A_M(IJK,east)
 * and A_M(IP_OF(IJK),west)); restated as a gather per fluid cell, it is
 * A(west) = ROP_GE(IMJK)*AYZ(IMJK) whether or not IMJK is fluid (:80-106).
 * Every sum keeps the reference's left-to-right order. */
static int fluid_at(const int *flag, int64_t p) { return flag[p] == 1; }
static int p_flow_at(const int *flag, int64_t p) { return flag[p] == 10 || flag[p] == 11; }

void orc_conv_source_pp_g(const orc_geom *g, const orc_pp_fields *f, double *a, double *b, double *bmmax)
{
    const int64_t n = g->n, c1 = g->jmax2, c2 = (int64_t)g->jmax2 * g->imax2;
    double *am3 = a, *am2 = a + n, *am1 = a + 2 * n, *a0 = a + 3 * n, *ap1 = a + 4 * n, *ap2 = a + 5 * n,
           *ap3 = a + 6 * n;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= g->kmax2; ++k)
        for (int i = 1; i <= g->imax2; ++i)
            for (int j = 1; j <= g->jmax2; ++j) {
                const int64_t p = cell(g, i, j, k);
                if (!fluid_at(f->flag, p)) {  /* :187-199 */
                    am3[p] = am2[p] = am1[p] = ap1[p] = ap2[p] = ap3[p] = 0.0;
                    a0[p] = -1.0;
                    b[p] = 0.0;
                    bmmax[p] = 0.0;
                    continue;
                }
                /* clamped neighbours (model/set_increments.f:80-109) */
                const int64_t im = p + (i > 1 ? -c1 : 0), ip = p + (i < g->imax2 ? c1 : 0);
                const int64_t jm = p + (j > 1 ? -1 : 0), jp = p + (j < g->jmax2 ? 1 : 0);
                const int64_t km = p + ((g->do_k && k > 1) ? -c2 : 0), kp = p + ((g->do_k && k < g->kmax2) ? c2 : 0);
                /* CONV_PP_G, gas phase (:80-119) */
                double ae = f->rop_ge[p] * f->ayz[p];
                double aw = f->rop_ge[im] * f->ayz[im];
                double an = f->rop_gn[p] * f->axz[p];
                double as = f->rop_gn[jm] * f->axz[jm];
                double at = 0.0, ab = 0.0;
                if (g->do_k) {
                    at = f->rop_gt[p] * f->axy[p];
                    ab = f->rop_gt[km] * f->axy[km];
                }
                /* SOURCE_PP_G (:87-106) */
                const double bma = (f->rop_g[p] - f->rop_go[p]) * f->vol[p] * f->odt;
                const double bme = ae * f->u_g[p];
                const double bmw = aw * f->u_g[im];
                const double bmn = an * f->v_g[p];
                const double bms = as * f->v_g[jm];
                const double bmt = g->do_k ? at * f->w_g[p] : 0.0;
                const double bmb = g->do_k ? ab * f->w_g[km] : 0.0;
                const double bmr = f->sum_r_g[p] * f->vol[p];
                double bv = -((-(bma + bme - bmw + bmn - bms + bmt - bmb)) + bmr);
                double mx = fabs(bma);
                const double terms[7] = {bme, bmw, bmn, bms, bmt, bmb, bmr};
                for (int q = 0; q < 7; ++q)
                    if (fabs(terms[q]) > mx) mx = fabs(terms[q]);
                ae = ae * f->d_e[p];
                aw = aw * f->d_e[im];
                an = an * f->d_n[p];
                as = as * f->d_n[jm];
                if (g->do_k) {
                    at = at * f->d_t[p];
                    ab = ab * f->d_t[km];
                }
                /* solids phases that do not become close packed (:117-145; CONV_PP_G :125-178) */
                for (int m = 1; m <= f->mmax; ++m) {
                    if (f->close_packed[m - 1]) continue;
                    const int64_t o = (int64_t)(m - 1) * n, od = (int64_t)m * n;
                    const double se = f->rop_se[o + p] * f->ayz[p];
                    const double sw = f->rop_se[o + im] * f->ayz[im];
                    const double sn = f->rop_sn[o + p] * f->axz[p];
                    const double ss = f->rop_sn[o + jm] * f->axz[jm];
                    double st = 0.0, sb = 0.0;
                    if (g->do_k) {
                        st = f->rop_st[o + p] * f->axy[p];
                        sb = f->rop_st[o + km] * f->axy[km];
                    }
                    const double wt = g->do_k ? st * f->w_s[o + p] : 0.0;
                    const double wb = g->do_k ? sb * f->w_s[o + km] : 0.0;
                    bv = bv - ((-((f->rop_s[o + p] - f->rop_so[o + p]) * f->vol[p] * f->odt + se * f->u_s[o + p] -
                                   sw * f->u_s[o + im] + sn * f->v_s[o + p] - ss * f->v_s[o + jm] + wt - wb)) +
                               f->sum_r_s[o + p] * f->vol[p]);
                    ae = ae + se * f->d_e[od + p];
                    aw = aw + sw * f->d_e[od + im];
                    an = an + sn * f->d_n[od + p];
                    as = as + ss * f->d_n[od + jm];
                    if (g->do_k) {
                        at = at + st * f->d_t[od + p];
                        ab = ab + sb * f->d_t[od + km];
                    }
                }
                double ac = -(ae + aw + an + as + at + ab); /* :147-149 */
                if (fabs(ac) < 1.0e-15) {                    /* :151-162, SMALL_NUMBER */
                    if (fabs(bv) < 1.0e-15) {
                        ac = -1.0;
                        bv = 0.0;
                    }
                }
                /* links to pressure-flow cells cut (:224-243) */
                if (p_flow_at(f->flag, im)) aw = 0.0;
                if (p_flow_at(f->flag, ip)) ae = 0.0;
                if (p_flow_at(f->flag, jm)) as = 0.0;
                if (p_flow_at(f->flag, jp)) an = 0.0;
                if (p_flow_at(f->flag, km)) ab = 0.0;
                if (p_flow_at(f->flag, kp)) at = 0.0;
                am3[p] = ab;
                am2[p] = as;
                am1[p] = aw;
                a0[p] = ac;
                ap1[p] = ae;
                ap2[p] = an;
                ap3[p] = at;
                b[p] = bv;
                bmmax[p] = mx;
            }
    /* the reference cell of an incompressible run (:247-251) */
    if (f->ijk_p_g >= 1 && f->ijk_p_g <= n) {
        const int64_t p = f->ijk_p_g - 1;
        for (int q = 0; q < 7; ++q) a[q * n + p] = 0.0;
        a0[p] = -1.0;
        b[p] = 0.0;
    }
}

double orc_calc_resid_pp(const orc_geom *g, const int *flag, const double *b, double norm)
{
    double num = 0.0, den = 0.0;
    for (int64_t p = 0; p < g->n; ++p)
        if (fluid_at(flag, p)) {
            num = num + fabs(b[p]);
            den = den + 1.0;
        }
    if (den * norm > 0.0) return num / (den * norm);
    if (num == 0.0) return 0.0;
    return 1.0e32; /* LARGE_NUMBER */
}

/* ------------------------------------------------------------------ DO_TRANSPOSE: LEQ_BICGSt */
/* LEQ_MSOLVEt (model/leq_bicgst.f:978-1177): SETGUESS, then per letter: in 2-D
 * only I (LEQ_ISWEEPt over i in order); in 3-D R in the loop order of
 * :1040-1061 (two passes over ik = icase, icase+2, ...; i wraps within the row
 * when the row length is odd), I (k outer, i inner) and K (i outer, k inner).
 * A, J and S do nothing.  The line solves are LEQ_IKSWEEP's / LEQ_ISWEEP's on the
 * transposed copy, the same values. */
static int msolve_t(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep, int *skips)
{
    int nskip = 0;
    memcpy(var, b, sizeof(double) * (size_t)g->n);
    for (int it = 0; it < 4; ++it) {
        const char ch = sweep[it];
        const int do_i = (ch == 'I' || ch == 'i'), do_kk = (ch == 'K' || ch == 'k'), do_rb = (ch == 'R' || ch == 'r');
        if (!g->do_k) {
            if (do_i)
                for (int i = 1; i <= g->imax2; ++i) nskip += orc_isweep(g, i, var, a, b) != 0;
            continue;
        }
        if (do_rb) {
            const int i1 = 1, k1 = 1, i2 = g->imax2, k2 = g->kmax2, isize = i2 - i1 + 1, ksize = k2 - k1 + 1;
            for (int icase = 1; icase <= 2; ++icase)
                for (int ik = icase; ik <= ksize * isize; ik += 2) {
                    const int k = (ik % isize != 0) ? ik / isize + k1 : ik / isize + k1 - 1;
                    int i = (ik - 1 - (k - k1) * isize) + i1 + (k % 2);
                    if (i > i2) i = i - i2 + i1 - 1;
                    nskip += orc_iksweep(g, i, k, var, a, b) != 0;
                }
        }
        if (do_i)
            for (int k = 1; k <= g->kmax2; ++k)
                for (int i = 1; i <= g->imax2; ++i) nskip += orc_iksweep(g, i, k, var, a, b) != 0;
        if (do_kk)
            for (int i = 1; i <= g->imax2; ++i)
                for (int k = 1; k <= g->kmax2; ++k) nskip += orc_iksweep(g, i, k, var, a, b) != 0;
    }
    if (skips) *skips += nskip;
    return 0;
}

int orc_msolve_t(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep, int *skips)
{
    return msolve_t(g, b, a, var, sweep, skips);
}

int orc_leq_bicgst(const orc_geom *g, double *var, const double *a, double *b, const char *sweep, double tol,
                   const char *pc, int itmax, uint64_t rt_seed, int minimize, orc_stats *st)
{
    /* SOLVE_LIN_EQ's transposed copy A_mt (model/solve_lin_eq.f:139-150): scaled, then discarded */
    double *at = (double *)malloc(sizeof(double) * 7 * (size_t)g->n);
    memcpy(at, a, sizeof(double) * 7 * (size_t)g->n);
    const int r = bicgs_run_x(g, var, at, b, sweep, tol, pc, itmax, rt_seed, -1, st, 1, minimize ? 5 : 0);
    free(at);
    return r;
}
