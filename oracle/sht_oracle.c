/*
 * sht_oracle.c -- CPU FP64 restatement of dogcm's horizontal spherical-
 * harmonic transform (the SpmlUtil_mod -> SPMODEL wa_module path).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
 * and the timed CPU baseline; nothing in the product links or calls it.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The
 * reference keeps the arithmetic in the external SPMODEL (>=0.8.0) and
 * ISPACK (1.0.4) libraries, which are not vendored in the reference tree,
 * and the reference has no test or golden file for this transform.  This
 * restatement follows the written specification in the reference:
 *
 *   doc/description/ogcm/space_discretization.tex:17-40   grid (lambda_i, Gauss mu_j ascending)
 *   doc/description/ogcm/space_discretization.tex:161-222 transform + normalisation
 *                                                        (P normalised to 2, w_j = 1/2 int ..., G^m = 1/I sum)
 *   doc/description/ogcm/space_discretization.tex:230-267 derivative transforms, recurrence
 *                                                        (1-mu^2) dP/dmu, operator H
 *   doc/description/ogcm/space_discretization.tex:350-381 psi/chi -> U, V
 *   model/dogcm/src/util/math/SpmlUtil_mod.f90:299-473    composites (1/a, 1/cos^2 factors)
 *   model/dogcm/src/physics/lphys/LPhys_DIFF_spm_mod.f90:144-158 diffusion coefficients
 *
 * and is checked against an independent scipy/numpy evaluation of the same
 * formulas (tests/golden/make_golden.py).
 *
 * Storage conventions (fixed here; the in-tree pins they satisfy are cited):
 *   grid   xy[j*I + i]  = Fortran xy(0:I-1, 1:J); lambda_i = 2 pi i / I,
 *          mu_j ascending from the south pole (space_discretization.tex:33-38).
 *   spectral w[l], l = n(n+1) + m  (0-based; Fortran l_nm(n,m) = n(n+1)+m+1,
 *          so l=1 is (0,0): HBEBarot_hspm_vfvm_mod.f90:295-298), m in [-n, n].
 *          w(n,0) = a_n^0, and for m > 0  w(n,m) = sqrt2 Re a_n^m,
 *          w(n,-m) = sqrt2 Im a_n^m, where the field is
 *          q = sum_n sum_{m=-n..n} a_n^m Pbar_n^|m|(mu) e^{i m lambda}
 *          (space_discretization.tex:161-170).  A unit real coefficient at
 *          m != 0 therefore has sqrt2 times the amplitude of an m = 0 mode,
 *          which is why the experiments scale by 1/sqrt2
 *          (exp/BarotRossby/DOGCM_Exp_BarotRossby_mod.f90:121-123).
 *   Pbar_n^m: int_{-1}^{1} Pbar^2 dmu = 2, no Condon-Shortley phase.
 *   y_Lat_Weight sums to 2 and x_Lon_Weight = 2 pi / I (cell widths in mu
 *          and lambda: seaice/admin/DSIce_Admin_GaussSpmGrid_mod.f90:325,
 *          seaice/dynamics/DSIce_Dyn_fvm_mod.f90:261).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_SQRT2 1.41421356237309504880

typedef struct {
    int I, J, N, JH, NC;  /* NC = I/2 when I is a power of two, else 0 */
    double radius;
    double *mu, *wgt, *coslat; /* wgt normalised to sum 1 */
    double *P;                 /* P[poff[m] + (n-m)*JH + jh], n = m..N+1, northern rows */
    long *poff;
    double *eps;               /* eps[m*(N+3) + n], n = 0..N+2 */
    double *tw_nc;             /* complex exp(-2 pi i k / NC), k < NC (re,im pairs) */
    double *tw_i;              /* complex exp(-2 pi i k / I),  k < I  (re,im pairs) */
    int *bitrev;               /* NC entries */
} or_plan;

/* ---------------------------------------------------------------- grid */

/* Gauss-Legendre nodes (ascending) and weights normalised to sum 1:
 * w_j = 1/2 int P_J/((mu-mu_j) P_J'(mu_j)) dmu  (space_discretization.tex:205-209).
 * Newton iteration on P_J with the three-term recurrence. */
int or_gauss(int J, double *mu, double *w)
{
    if (J < 1) return 1;
    for (int k = 0; k < (J + 1) / 2; ++k) {
        double x = cos(M_PI * (k + 0.75) / (J + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int n = 2; n <= J; ++n) {
                double p2 = ((2.0 * n - 1.0) * x * p1 - (n - 1.0) * p0) / n;
                p0 = p1; p1 = p2;
            }
            if (J == 1) { p1 = x; p0 = 1.0; }
            dp = J * (x * p1 - p0) / (x * x - 1.0);
            double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) < 1e-16 * (1.0 + fabs(x)) && it > 2) {
                /* one more evaluation for the derivative at the converged root */
                p0 = 1.0; p1 = x;
                for (int n = 2; n <= J; ++n) {
                    double p2 = ((2.0 * n - 1.0) * x * p1 - (n - 1.0) * p0) / n;
                    p0 = p1; p1 = p2;
                }
                dp = J * (x * p1 - p0) / (x * x - 1.0);
                break;
            }
        }
        double wk = 1.0 / ((1.0 - x * x) * dp * dp); /* = (2/((1-x^2)P'^2)) / 2 */
        /* x is the k-th largest root: store ascending */
        mu[J - 1 - k] = x;
        mu[k] = -x;
        w[J - 1 - k] = wk;
        w[k] = wk;
    }
    if (J % 2 == 1) mu[J / 2] = 0.0;
    return 0;
}

/* ---------------------------------------------------------------- FFT */

static int ilog2_exact(int n)
{
    int l = 0;
    if (n <= 0) return -1;
    while ((1 << l) < n) ++l;
    return ((1 << l) == n) ? l : -1;
}

/* in-place radix-2 complex DFT of size NC, sign -1 (forward) or +1. */
static void or_cfft(const or_plan *p, double *z, int sign)
{
    int nc = p->NC;
    for (int k = 0; k < nc; ++k) {
        int r = p->bitrev[k];
        if (r > k) {
            double t0 = z[2 * k], t1 = z[2 * k + 1];
            z[2 * k] = z[2 * r]; z[2 * k + 1] = z[2 * r + 1];
            z[2 * r] = t0; z[2 * r + 1] = t1;
        }
    }
    for (int len = 2; len <= nc; len <<= 1) {
        int half = len >> 1, step = nc / len;
        for (int s = 0; s < nc; s += len) {
            for (int k = 0; k < half; ++k) {
                /* tw_nc holds exp(-2 pi i k/NC); the inverse uses its conjugate */
                double wr = p->tw_nc[2 * (k * step)];
                double wi = (sign < 0) ? p->tw_nc[2 * (k * step) + 1] : -p->tw_nc[2 * (k * step) + 1];
                double *a = z + 2 * (s + k), *b = z + 2 * (s + k + half);
                double br = b[0] * wr - b[1] * wi, bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br; b[1] = a[1] - bi;
                a[0] += br; a[1] += bi;
            }
        }
    }
}

/* G^m = (1/I) sum_i x_i e^{-i m lambda_i}, m = 0..N  (space_discretization.tex:190-193).
 * out: G[2m], G[2m+1]. work: 2*I doubles. */
static void or_fourier_fwd(const or_plan *p, const double *x, double *G, double *work)
{
    int I = p->I, N = p->N;
    if (p->NC) {
        int nc = p->NC;
        for (int k = 0; k < nc; ++k) { work[2 * k] = x[2 * k]; work[2 * k + 1] = x[2 * k + 1]; }
        or_cfft(p, work, -1);
        for (int m = 0; m <= N; ++m) {
            int mm = (nc - m) % nc;
            double zr = work[2 * m], zi = work[2 * m + 1];
            double cr = work[2 * mm], ci = -work[2 * mm + 1]; /* conj Z_{NC-m} */
            double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
            double dr = 0.5 * (zr - cr), di = 0.5 * (zi - ci);
            double wr = p->tw_i[2 * m], wi = p->tw_i[2 * m + 1];
            /* X = E - i W D */
            double tr = wr * dr - wi * di, ti = wr * di + wi * dr;
            G[2 * m] = (er + ti) / I;
            G[2 * m + 1] = (ei - tr) / I;
        }
    } else {
        for (int m = 0; m <= N; ++m) {
            double sr = 0.0, si = 0.0;
            for (int i = 0; i < I; ++i) {
                long k = ((long)m * i) % I;
                sr += x[i] * p->tw_i[2 * k];
                si += x[i] * p->tw_i[2 * k + 1];
            }
            G[2 * m] = sr / I;
            G[2 * m + 1] = si / I;
        }
    }
    G[1] = 0.0;
}

/* x_i = sum_{m=-N..N} G^m e^{i m lambda_i} with G^{-m} = conj G^m
 * (space_discretization.tex:217-222). work: 2*I doubles. */
static void or_fourier_inv(const or_plan *p, const double *G, double *x, double *work)
{
    int I = p->I, N = p->N;
    if (p->NC) {
        int nc = p->NC;
        for (int k = 0; k < nc; ++k) {
            double xr = 0, xi = 0, yr = 0, yi = 0; /* X_k and X_{k+NC} */
            if (k <= N) { xr = G[2 * k]; xi = (k == 0) ? 0.0 : G[2 * k + 1]; }
            int km = nc - k; /* X_{k+NC} = conj X_{NC-k} */
            if (k > 0 && km <= N) { yr = G[2 * km]; yi = -G[2 * km + 1]; }
            double wr = p->tw_i[2 * k], wi = -p->tw_i[2 * k + 1]; /* e^{+2 pi i k/I} */
            double dr = xr - yr, di = xi - yi;
            /* Z = (X + Y) + i w (X - Y) */
            double tr = wr * dr - wi * di, ti = wr * di + wi * dr;
            work[2 * k] = (xr + yr) - ti;
            work[2 * k + 1] = (xi + yi) + tr;
        }
        or_cfft(p, work, +1);
        for (int k = 0; k < nc; ++k) { x[2 * k] = work[2 * k]; x[2 * k + 1] = work[2 * k + 1]; }
    } else {
        for (int i = 0; i < I; ++i) {
            double s = G[0];
            for (int m = 1; m <= N; ++m) {
                long k = ((long)m * i) % I;
                /* e^{+i m lambda} = conj(tw_i[k]) */
                double cr = p->tw_i[2 * k], ci = -p->tw_i[2 * k + 1];
                s += 2.0 * (G[2 * m] * cr - G[2 * m + 1] * ci);
            }
            x[i] = s;
        }
    }
}

/* ------------------------------------------------------------- Legendre */

/* Pbar_n^m at the northern Gauss rows, n = m..N+1, by the normalised
 * three-term recurrence mu P_n = eps_{n+1} P_{n+1} + eps_n P_{n-1},
 * eps_n^m = sqrt((n^2-m^2)/(4n^2-1)) (space_discretization.tex:250-257). */
static void or_build_legendre(or_plan *p)
{
    int N = p->N, JH = p->JH, J = p->J;
    for (int m = 0; m <= N; ++m)
        for (int n = 0; n <= N + 2; ++n)
            p->eps[m * (N + 3) + n] = (n < m || n == 0) ? 0.0 : sqrt(((double)n * n - (double)m * m) / (4.0 * n * n - 1.0));
    for (int jh = 0; jh < JH; ++jh) {
        double x = p->mu[J - JH + jh];
        double s = sqrt(1.0 - x * x);
        double pmm = 1.0;
        for (int m = 0; m <= N; ++m) {
            if (m > 0) pmm *= sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
            double *col = p->P + p->poff[m];
            double pm2 = 0.0, pm1 = pmm;
            col[jh] = pmm;
            for (int n = m + 1; n <= N + 1; ++n) {
                double e_n = p->eps[m * (N + 3) + n], e_nm1 = p->eps[m * (N + 3) + n - 1];
                double pn = (x * pm1 - e_nm1 * pm2) / e_n;
                col[(long)(n - m) * JH + jh] = pn;
                pm2 = pm1; pm1 = pn;
            }
        }
    }
}

/* c_n^m = sum_j w_j G^m(mu_j) Pbar_n^m(mu_j), n = m..N+1, per m
 * (space_discretization.tex:197-200), using Pbar(-mu) = (-1)^{n-m} Pbar(mu).
 * G: [j][m] complex.  c: [coff(m) + (n-m)] complex, coff(m) = sum_{m'<m}(N+2-m'). */
static void or_legendre_fwd(const or_plan *p, const double *G, double *c, double *work)
{
    int N = p->N, J = p->J, JH = p->JH;
    double *gs = work, *ga = work + 2 * JH;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        for (int jh = 0; jh < JH; ++jh) {
            int jn = J - JH + jh, js = JH - 1 - jh;
            double w = p->wgt[jn];
            const double *a = G + 2 * ((long)jn * (N + 1) + m), *b = G + 2 * ((long)js * (N + 1) + m);
            gs[2 * jh] = w * (a[0] + b[0]); gs[2 * jh + 1] = w * (a[1] + b[1]);
            ga[2 * jh] = w * (a[0] - b[0]); ga[2 * jh + 1] = w * (a[1] - b[1]);
        }
        const double *col = p->P + p->poff[m];
        for (int n = m; n <= N + 1; ++n) {
            const double *g = ((n - m) & 1) ? ga : gs;
            const double *pr = col + (long)(n - m) * JH;
            double sr = 0.0, si = 0.0;
            for (int jh = 0; jh < JH; ++jh) { sr += pr[jh] * g[2 * jh]; si += pr[jh] * g[2 * jh + 1]; }
            c[2 * (co + n - m)] = sr;
            c[2 * (co + n - m) + 1] = si;
        }
        co += N + 2 - m;
    }
}

/* G^m(mu_j) = sum_n a_n^m Pbar_n^m(mu_j), n = m..N+1 (space_discretization.tex:212-216). */
static void or_legendre_inv(const or_plan *p, const double *a, double *G, double *work)
{
    int N = p->N, J = p->J, JH = p->JH;
    double *ge = work, *go = work + 2 * JH;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        memset(work, 0, sizeof(double) * 4 * JH);
        const double *col = p->P + p->poff[m];
        for (int n = m; n <= N + 1; ++n) {
            double ar = a[2 * (co + n - m)], ai = a[2 * (co + n - m) + 1];
            if (ar == 0.0 && ai == 0.0) continue;
            double *g = ((n - m) & 1) ? go : ge;
            const double *pr = col + (long)(n - m) * JH;
            for (int jh = 0; jh < JH; ++jh) { g[2 * jh] += pr[jh] * ar; g[2 * jh + 1] += pr[jh] * ai; }
        }
        for (int jh = 0; jh < JH; ++jh) {
            int jn = J - JH + jh, js = JH - 1 - jh;
            double *x = G + 2 * ((long)jn * (N + 1) + m), *y = G + 2 * ((long)js * (N + 1) + m);
            x[0] = ge[2 * jh] + go[2 * jh]; x[1] = ge[2 * jh + 1] + go[2 * jh + 1];
            y[0] = ge[2 * jh] - go[2 * jh]; y[1] = ge[2 * jh + 1] - go[2 * jh + 1];
        }
        co += N + 2 - m;
    }
}

/* ------------------------------------------------------------- plan */

or_plan *or_init(int I, int J, int N, double radius)
{
    if (I < 1 || J < 2 || (J & 1) || N < 0 || I < 2 * N + 1 || J <= N) return NULL;
    or_plan *p = (or_plan *)calloc(1, sizeof(or_plan));
    p->I = I; p->J = J; p->N = N; p->JH = J / 2; p->radius = radius;
    p->NC = (ilog2_exact(I) >= 1) ? I / 2 : 0;
    p->mu = (double *)malloc(sizeof(double) * J);
    p->wgt = (double *)malloc(sizeof(double) * J);
    p->coslat = (double *)malloc(sizeof(double) * J);
    or_gauss(J, p->mu, p->wgt);
    for (int j = 0; j < J; ++j) p->coslat[j] = sqrt(1.0 - p->mu[j] * p->mu[j]);
    p->poff = (long *)malloc(sizeof(long) * (N + 2));
    long off = 0;
    for (int m = 0; m <= N; ++m) { p->poff[m] = off; off += (long)(N + 2 - m) * p->JH; }
    p->poff[N + 1] = off;
    p->P = (double *)malloc(sizeof(double) * (off > 0 ? off : 1));
    p->eps = (double *)malloc(sizeof(double) * (N + 1) * (N + 3));
    or_build_legendre(p);
    p->tw_i = (double *)malloc(sizeof(double) * 2 * I);
    for (int k = 0; k < I; ++k) {
        long double t = -2.0L * 3.141592653589793238462643383279502884L * k / I;
        p->tw_i[2 * k] = (double)cosl(t);
        p->tw_i[2 * k + 1] = (double)sinl(t);
    }
    if (p->NC) {
        int nc = p->NC, lg = ilog2_exact(nc);
        p->tw_nc = (double *)malloc(sizeof(double) * 2 * nc);
        p->bitrev = (int *)malloc(sizeof(int) * nc);
        for (int k = 0; k < nc; ++k) {
            long double t = -2.0L * 3.141592653589793238462643383279502884L * k / nc;
            p->tw_nc[2 * k] = (double)cosl(t);
            p->tw_nc[2 * k + 1] = (double)sinl(t);
            int r = 0;
            for (int b = 0; b < lg; ++b) if (k & (1 << b)) r |= 1 << (lg - 1 - b);
            p->bitrev[k] = r;
        }
    }
    return p;
}

void or_free(or_plan *p)
{
    if (!p) return;
    free(p->mu); free(p->wgt); free(p->coslat); free(p->P); free(p->poff);
    free(p->eps); free(p->tw_i); free(p->tw_nc); free(p->bitrev);
    free(p);
}

long or_lm(const or_plan *p) { return (long)(p->N + 1) * (p->N + 1); }
long or_ncoef_ext(const or_plan *p) { return (long)(p->N + 1) * (p->N + 4) / 2; }

/* get_SpmlGridInfo (SpmlUtil_mod.f90:271-295): x_Lon, y_Lat (radians),
 * x_Lon_Weight (sum 2 pi), y_Lat_Weight (sum 2). */
void or_grid_info(const or_plan *p, double *x_lon, double *y_lat, double *x_w, double *y_w)
{
    for (int i = 0; i < p->I; ++i) {
        if (x_lon) x_lon[i] = 2.0 * M_PI * i / p->I;
        if (x_w) x_w[i] = 2.0 * M_PI / p->I;
    }
    for (int j = 0; j < p->J; ++j) {
        if (y_lat) y_lat[j] = asin(p->mu[j]);
        if (y_w) y_w[j] = 2.0 * p->wgt[j];
    }
}

void or_gauss_table(const or_plan *p, double *mu, double *w) { memcpy(mu, p->mu, sizeof(double) * p->J); memcpy(w, p->wgt, sizeof(double) * p->J); }

/* the Legendre table row Pbar_n^m at northern rows (for tests) */
void or_legendre_row(const or_plan *p, int n, int m, double *out)
{
    memcpy(out, p->P + p->poff[m] + (long)(n - m) * p->JH, sizeof(double) * p->JH);
}

/* l_nm / nm_l with Fortran 1-based l */
int or_l_nm(int n, int m) { return n * (n + 1) + m + 1; }
void or_nm_l(int l, int *n, int *m)
{
    int nn = (int)floor(sqrt((double)(l - 1)));
    while ((nn + 1) * (nn + 1) <= l - 1) ++nn;
    while (nn * nn > l - 1) --nn;
    *n = nn; *m = (l - 1) - nn * (nn + 1);
}

/* ------------------------------------------------------ spectral helpers */

static double eps_at(const or_plan *p, int m, int n) { return (n < 0 || n > p->N + 2) ? 0.0 : p->eps[m * (p->N + 3) + n]; }

/* SPML layout -> complex a_n^m, n = m..N+1 (a_{N+1} = 0) */
static void unpack(const or_plan *p, const double *w, double *a)
{
    int N = p->N;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        for (int n = m; n <= N + 1; ++n) {
            double re = 0, im = 0;
            if (n <= N) {
                if (m == 0) re = w[n * (n + 1)];
                else { re = w[n * (n + 1) + m] / OR_SQRT2; im = w[n * (n + 1) - m] / OR_SQRT2; }
            }
            a[2 * (co + n - m)] = re; a[2 * (co + n - m) + 1] = im;
        }
        co += N + 2 - m;
    }
}

static void pack(const or_plan *p, const double *c, double *w)
{
    int N = p->N;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        for (int n = m; n <= N; ++n) {
            double re = c[2 * (co + n - m)], im = c[2 * (co + n - m) + 1];
            if (m == 0) w[n * (n + 1)] = re;
            else { w[n * (n + 1) + m] = OR_SQRT2 * re; w[n * (n + 1) - m] = OR_SQRT2 * im; }
        }
        co += N + 2 - m;
    }
}

/* a -> i m a */
static void times_im(const or_plan *p, double *a)
{
    int N = p->N;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        for (int r = 0; r < N + 2 - m; ++r) {
            double re = a[2 * (co + r)], im = a[2 * (co + r) + 1];
            a[2 * (co + r)] = -m * im; a[2 * (co + r) + 1] = m * re;
        }
        co += N + 2 - m;
    }
}

/* synthesis side of (1-mu^2) d/dmu: coefficients b_k of Pbar_k, k = m..N+1,
 * b_k = (k+2) eps_{k+1} a_{k+1} - (k-1) eps_k a_{k-1}
 * (recurrence at space_discretization.tex:250-252; same form as the U,V
 * formula at :369-379). */
static void gradmu_coef(const or_plan *p, const double *a, double *b)
{
    int N = p->N;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        int len = N + 2 - m;
        for (int r = 0; r < len; ++r) {
            int k = m + r;
            double br = 0, bi = 0;
            if (r + 1 < len) { double e = (k + 2) * eps_at(p, m, k + 1); br += e * a[2 * (co + r + 1)]; bi += e * a[2 * (co + r + 1) + 1]; }
            if (r >= 1) { double e = (k - 1) * eps_at(p, m, k); br -= e * a[2 * (co + r - 1)]; bi -= e * a[2 * (co + r - 1) + 1]; }
            b[2 * (co + r)] = br; b[2 * (co + r) + 1] = bi;
        }
        co += len;
    }
}

/* analysis side: d = -( (n+1) eps_n c_{n-1} - n eps_{n+1} c_{n+1} ), n = m..N
 * i.e. -sum_j w_j G/(1-mu^2) (1-mu^2) dPbar/dmu (space_discretization.tex:262-267,
 * by parts, with B = 0 at the poles). */
static void divmu_coef(const or_plan *p, const double *c, double *d)
{
    int N = p->N;
    long co = 0;
    for (int m = 0; m <= N; ++m) {
        int len = N + 2 - m;
        for (int r = 0; r < len; ++r) {
            int n = m + r;
            double dr = 0, di = 0;
            if (n <= N) {
                if (r >= 1) { double e = (n + 1) * eps_at(p, m, n); dr -= e * c[2 * (co + r - 1)]; di -= e * c[2 * (co + r - 1) + 1]; }
                { double e = n * eps_at(p, m, n + 1); dr += e * c[2 * (co + r + 1)]; di += e * c[2 * (co + r + 1) + 1]; }
            }
            d[2 * (co + r)] = dr; d[2 * (co + r) + 1] = di;
        }
        co += len;
    }
}

/* ------------------------------------------------- per-field-level ops */

typedef struct { double *G, *c, *c2, *work; } or_ws;

static or_ws ws_alloc(const or_plan *p)
{
    or_ws w;
    long nce = or_ncoef_ext(p);
    w.G = (double *)malloc(sizeof(double) * 2 * (long)p->J * (p->N + 1));
    w.c = (double *)malloc(sizeof(double) * 2 * nce);
    w.c2 = (double *)malloc(sizeof(double) * 2 * nce);
    w.work = (double *)malloc(sizeof(double) * (4 * (long)p->I + 4 * (long)p->J + 16));
    return w;
}
static void ws_free(or_ws *w) { free(w->G); free(w->c); free(w->c2); free(w->work); }

enum { RS_NONE = 0, RS_INV1MMU2 = 1, RS_INVCOS = 2, RS_COS = 3 };
static double rowscale(const or_plan *p, int kind, int j)
{
    double mu = p->mu[j];
    switch (kind) {
    case RS_INV1MMU2: return 1.0 / (1.0 - mu * mu);
    case RS_INVCOS: return 1.0 / p->coslat[j];
    case RS_COS: return p->coslat[j];
    default: return 1.0;
    }
}

/* grid -> c (extended, n = m..N+1), optional row scale applied to the grid */
static void analysis_ext(const or_plan *p, const double *xy, int rs, or_ws *w, double *c)
{
    int I = p->I, N = p->N;
    double *row = w->work + 2 * (long)I + 8;
    for (int j = 0; j < p->J; ++j) {
        double s = rowscale(p, rs, j);
        for (int i = 0; i < I; ++i) row[i] = xy[(long)j * I + i] * s;
        or_fourier_fwd(p, row, w->G + 2 * (long)j * (N + 1), w->work);
    }
    or_legendre_fwd(p, w->G, c, w->work);
}

static void synthesis_ext(const or_plan *p, const double *a, int rs, or_ws *w, double *xy)
{
    int I = p->I, N = p->N;
    or_legendre_inv(p, a, w->G, w->work);
    for (int j = 0; j < p->J; ++j) {
        or_fourier_inv(p, w->G + 2 * (long)j * (N + 1), xy + (long)j * I, w->work);
        double s = rowscale(p, rs, j);
        if (rs != RS_NONE) for (int i = 0; i < I; ++i) xy[(long)j * I + i] *= s;
    }
}

/* w_xy */
static void op_w_xy(const or_plan *p, const double *xy, double *wout, or_ws *w)
{ analysis_ext(p, xy, RS_NONE, w, w->c); pack(p, w->c, wout); }

/* xy_w */
static void op_xy_w(const or_plan *p, const double *win, double *xy, or_ws *w)
{ unpack(p, win, w->c); synthesis_ext(p, w->c, RS_NONE, w, xy); }

/* w_DivLambda_xy: spectral of 1/(1-mu^2) dA/dlambda */
static void op_divlambda(const or_plan *p, const double *xy, double *wout, or_ws *w)
{ analysis_ext(p, xy, RS_INV1MMU2, w, w->c); times_im(p, w->c); pack(p, w->c, wout); }

/* w_DivMu_xy: spectral of dB/dmu */
static void op_divmu(const or_plan *p, const double *xy, double *wout, or_ws *w)
{ analysis_ext(p, xy, RS_INV1MMU2, w, w->c); divmu_coef(p, w->c, w->c2); pack(p, w->c2, wout); }

/* xy_GradLambda_w: d/dlambda */
static void op_gradlambda(const or_plan *p, const double *win, double *xy, int rs, or_ws *w)
{ unpack(p, win, w->c); times_im(p, w->c); synthesis_ext(p, w->c, rs, w, xy); }

/* xy_GradMu_w: (1-mu^2) d/dmu */
static void op_gradmu(const or_plan *p, const double *win, double *xy, int rs, or_ws *w)
{ unpack(p, win, w->c); gradmu_coef(p, w->c, w->c2); synthesis_ext(p, w->c2, rs, w, xy); }

/* ------------------------------------------------------- batched API */

#define OR_BATCH(body) do { \
    _Pragma("omp parallel") { or_ws w_ = ws_alloc(p); \
    _Pragma("omp for schedule(static)") for (int b = 0; b < nb; ++b) { body; } \
    ws_free(&w_); } } while (0)

void or_wa_xya(const or_plan *p, const double *xya, int nb, double *wa)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_w_xy(p, xya + b * IJ, wa + b * L, &w_)); }

void or_xya_wa(const or_plan *p, const double *wa, int nb, double *xya)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_xy_w(p, wa + b * L, xya + b * IJ, &w_)); }

void or_wa_divlambda_xya(const or_plan *p, const double *xya, int nb, double *wa)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_divlambda(p, xya + b * IJ, wa + b * L, &w_)); }

void or_wa_divmu_xya(const or_plan *p, const double *xya, int nb, double *wa)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_divmu(p, xya + b * IJ, wa + b * L, &w_)); }

void or_xya_gradlambda_wa(const or_plan *p, const double *wa, int nb, double *xya)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_gradlambda(p, wa + b * L, xya + b * IJ, RS_NONE, &w_)); }

void or_xya_gradmu_wa(const or_plan *p, const double *wa, int nb, double *xya)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_gradmu(p, wa + b * L, xya + b * IJ, RS_NONE, &w_)); }

/* xy_GradLon_w = (1/cos phi) d/dlambda ; xy_GradLat_w = d/dphi = (1/cos phi)(1-mu^2) d/dmu
 * (SPMODEL definitions; used unscaled by the radius at
 * exp/BarotRossby/DOGCM_Exp_BarotRossby_mod.f90:125-126). */
void or_xya_gradlon_wa(const or_plan *p, const double *wa, int nb, double *xya)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_gradlambda(p, wa + b * L, xya + b * IJ, RS_INVCOS, &w_)); }

void or_xya_gradlat_wa(const or_plan *p, const double *wa, int nb, double *xya)
{ long IJ = (long)p->I * p->J, L = or_lm(p); OR_BATCH(op_gradmu(p, wa + b * L, xya + b * IJ, RS_INVCOS, &w_)); }

/* w_Lapla_w: rn(l,1) = -n(n+1) (LPhys_DIFF_spm_mod.f90:144) */
void or_wa_lapla_wa(const or_plan *p, const double *wa, int nb, double *out)
{
    long L = or_lm(p);
    for (int b = 0; b < nb; ++b)
        for (long l = 0; l < L; ++l) { int n, m; or_nm_l((int)l + 1, &n, &m); out[b * L + l] = -(double)n * (n + 1) * wa[b * L + l]; }
}

/* w_LaplaInv_w: 1/rn with the n = 0 mode set to zero */
void or_wa_laplainv_wa(const or_plan *p, const double *wa, int nb, double *out)
{
    long L = or_lm(p);
    for (int b = 0; b < nb; ++b)
        for (long l = 0; l < L; ++l) { int n, m; or_nm_l((int)l + 1, &n, &m); out[b * L + l] = (n == 0) ? 0.0 : -wa[b * L + l] / ((double)n * (n + 1)); }
}

void or_rn(const or_plan *p, double *rn)
{
    long L = or_lm(p);
    for (long l = 0; l < L; ++l) { int n, m; or_nm_l((int)l + 1, &n, &m); rn[l] = -(double)n * (n + 1); }
}

/* w_AlphaOptr_xy = (w_DivLambda_xy(A) + w_DivMu_xy(B)) / a  (SpmlUtil_mod.f90:398-412) */
void or_wa_alphaoptr_xya(const or_plan *p, const double *A, const double *B, int nb, double *out)
{
    long IJ = (long)p->I * p->J, L = or_lm(p);
    double *tmp = (double *)malloc(sizeof(double) * L * (nb > 0 ? nb : 1));
    or_wa_divlambda_xya(p, A, nb, out);
    or_wa_divmu_xya(p, B, nb, tmp);
    for (long k = 0; k < L * nb; ++k) out[k] = (out[k] + tmp[k]) / p->radius;
    free(tmp);
    (void)IJ;
}

/* xy_AlphaOptr_w = (xy_GradLambda_w(A) + xy_GradMu_w(B)) / (a cos^2 phi)  (SpmlUtil_mod.f90:414-428) */
void or_xya_alphaoptr_wa(const or_plan *p, const double *wA, const double *wB, int nb, double *out)
{
    long IJ = (long)p->I * p->J;
    double *tmp = (double *)malloc(sizeof(double) * IJ * (nb > 0 ? nb : 1));
    or_xya_gradlambda_wa(p, wA, nb, out);
    or_xya_gradmu_wa(p, wB, nb, tmp);
    for (int b = 0; b < nb; ++b)
        for (int j = 0; j < p->J; ++j) {
            double c = p->coslat[j];
            double s = 1.0 / (p->radius * c * c);
            for (int i = 0; i < p->I; ++i) { long k = b * IJ + (long)j * p->I + i; out[k] = (out[k] + tmp[k]) * s; }
        }
    free(tmp);
}

/* calc_UVCosLat2VorDiv (SpmlUtil_mod.f90:299-314):
 * Vor = w_AlphaOptr_xy(V cos, -U cos); Div = w_AlphaOptr_xy(U cos, V cos). */
void or_uvcoslat2vordiv(const or_plan *p, const double *U, const double *V, int nb, double *vor, double *div)
{
    long IJ = (long)p->I * p->J;
    double *mU = (double *)malloc(sizeof(double) * IJ * (nb > 0 ? nb : 1));
    for (long k = 0; k < IJ * nb; ++k) mU[k] = -U[k];
    or_wa_alphaoptr_xya(p, V, mU, nb, vor);
    or_wa_alphaoptr_xya(p, U, V, nb, div);
    free(mU);
}

/* calc_VorDiv2UV (SpmlUtil_mod.f90:316-340):
 * Psi = LaplaInv(Vor) a^2, Chi = LaplaInv(Div) a^2,
 * U = cos * xy_AlphaOptr_w(Chi, -Psi), V = cos * xy_AlphaOptr_w(Psi, Chi). */
void or_vordiv2uv(const or_plan *p, const double *vor, const double *div, int nb, double *U, double *V)
{
    long IJ = (long)p->I * p->J, L = or_lm(p);
    double *psi = (double *)malloc(sizeof(double) * L * (nb > 0 ? nb : 1));
    double *chi = (double *)malloc(sizeof(double) * L * (nb > 0 ? nb : 1));
    double *mpsi = (double *)malloc(sizeof(double) * L * (nb > 0 ? nb : 1));
    double a2 = p->radius * p->radius;
    or_wa_laplainv_wa(p, vor, nb, psi);
    or_wa_laplainv_wa(p, div, nb, chi);
    for (long k = 0; k < L * nb; ++k) { psi[k] *= a2; chi[k] *= a2; mpsi[k] = -psi[k]; }
    or_xya_alphaoptr_wa(p, chi, mpsi, nb, U);
    or_xya_alphaoptr_wa(p, psi, chi, nb, V);
    for (int b = 0; b < nb; ++b)
        for (int j = 0; j < p->J; ++j)
            for (int i = 0; i < p->I; ++i) { long k = b * IJ + (long)j * p->I + i; U[k] *= p->coslat[j]; V[k] *= p->coslat[j]; }
    free(psi); free(chi); free(mpsi);
}

/* IntLonLat_xy / AvrLonLat_xy: Gauss-weighted global integral and mean */
void or_intlonlat(const or_plan *p, const double *xya, int nb, double *out, int average)
{
    long IJ = (long)p->I * p->J;
    for (int b = 0; b < nb; ++b) {
        double s = 0.0;
        for (int j = 0; j < p->J; ++j) {
            double r = 0.0;
            for (int i = 0; i < p->I; ++i) r += xya[b * IJ + (long)j * p->I + i];
            s += r * (2.0 * M_PI / p->I) * (2.0 * p->wgt[j]);
        }
        out[b] = average ? s / (4.0 * M_PI) : s;
    }
}

/* ya_IntLon_xya / ya_AvrLon_xya: zonal integral and mean, out[b*J + j] */
void or_intlon(const or_plan *p, const double *xya, int nb, double *out, int average)
{
    long IJ = (long)p->I * p->J;
    for (int b = 0; b < nb; ++b)
        for (int j = 0; j < p->J; ++j) {
            double r = 0.0;
            for (int i = 0; i < p->I; ++i) r += xya[b * IJ + (long)j * p->I + i];
            out[(long)b * p->J + j] = average ? r / p->I : r * (2.0 * M_PI / p->I);
        }
}

/* Spectral backward-Euler lateral diffusion w <- filter w / (1 - dt c_l)
 * (DOGCM_Phys_hspm_vfvm_mod.f90:638-641, 741-742). */
void or_diffuse(const or_plan *p, double *wa, int nb, const double *coef, double dt, const double *filter)
{
    long L = or_lm(p);
    for (int b = 0; b < nb; ++b)
        for (long l = 0; l < L; ++l) {
            double f = filter ? filter[l] : 1.0;
            wa[b * L + l] = f * wa[b * L + l] / (1.0 - dt * coef[l]);
        }
}

/* Diffusion diagonals of LPhys_DIFF_spm_Init (LPhys_DIFF_spm_mod.f90:144-158):
 * ev = rn/a^2, c_trc = -(kh (-ev) + knum (-ev)^(ord/2)),
 * c_mom = -(nu (-ev - 2/a^2) + knum ((-ev)^(ord/2) - (2/a^2)^(ord/2))). */
void or_diffcoef(const or_plan *p, double diff, double visc, double numdiff, int ord, double *c_trc, double *c_mom)
{
    long L = or_lm(p);
    double a2 = p->radius * p->radius;
    for (long l = 0; l < L; ++l) {
        int n, m; or_nm_l((int)l + 1, &n, &m);
        double ev = -(double)n * (n + 1) / a2;
        if (c_trc) c_trc[l] = -(diff * (-ev) + numdiff * pow(-ev, ord / 2));
        if (c_mom) c_mom[l] = -(visc * (-ev - 2.0 / a2) + numdiff * (pow(-ev, ord / 2) - pow(2.0 / a2, ord / 2)));
    }
}

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
