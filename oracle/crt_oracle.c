/*
 * crt_oracle.c -- CPU FP64 restatement of the CRTomo hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity oracle and the timed CPU baseline.
 * Nothing in the shipped package links or calls this code.
 *
 * The reference (geophysics-ubonn/crtomo_stable) is Fortran 90 and cannot be
 * compiled in this environment (no Fortran compiler), so this file restates
 * each routine on the path loop by loop, in the reference's summation order,
 * with the reference's array layouts (column-major, 1-based indices held in
 * the integer arrays).  Each function cites the routine it follows.  Build
 * with -fcx-fortran-rules so that complex multiply / divide follow the same
 * rules gfortran uses.
 */
#include "crt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.141592653589793238462643383279502884

/* Fortran-layout accessors (1-based arguments). */
#define NREL(p, iel, k) ((p)->nrel[((size_t)(k) - 1) * ((p)->elanz + (p)->relanz) + (iel) - 1])
#define NMN(p) ((p)->maxnodes * ((p)->maxnodes + 1) / 2)
#define ELBG(p, iel, imn, ki) \
    ((p)->elbg[(((size_t)(ki) - 1) * NMN(p) + (imn) - 1) * (p)->elanz + (iel) - 1])
#define RELBG(p, rel, imn) ((p)->relbg[((size_t)(imn) - 1) * (p)->relanz + (rel) - 1])
#define KG(p, rel, l, ki) \
    ((p)->kg[(((size_t)(ki) - 1) * (p)->eanz + (l) - 1) * (p)->relanz + (rel) - 1])
#define KPOT(p, kp, j, l, ki) \
    ((kp)[(((size_t)(ki) - 1) * (p)->eanz + (l) - 1) * (p)->sanz + (j) - 1])
#define SX(p, node) ((p)->sx[(p)->snr[(node) - 1] - 1])
#define SY(p, node) ((p)->sy[(p)->snr[(node) - 1] - 1])

static inline int imax_i(int a, int b) { return a > b ? a : b; }
static inline int imin_i(int a, int b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* Quadrature: src/gauleg.f90:17-38 (Gauss-Legendre by Newton iteration on
 * the Legendre recurrence) and src/gaulag.f90:16-42 (Gauss-Laguerre). */
void orc_gauleg(double x1, double x2, double *x, double *w, int n)
{
    const double eps = 3.0e-14;
    int m = (n + 1) / 2;
    double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
    for (int i = 1; i <= m; ++i) {
        double z = cos(3.141592653589793 * ((double)i - 0.25) / ((double)n + 0.5));
        double z1, pp, p1, p2, p3;
        do {
            p1 = 1.0;
            p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
            }
            pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
        } while (fabs(z - z1) > eps);
        x[i - 1] = xm - xl * z;
        x[n - i] = xm + xl * z;
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
}

void orc_gaulag(double *x, double *w, int n, double alf)
{
    const double eps = 3.0e-14;
    const int maxit = 10;
    double z = 0.0, pp = 0.0, p1, p2 = 0.0, p3;
    for (int i = 1; i <= n; ++i) {
        if (i == 1) {
            z = (1.0 + alf) * (3.0 + 0.92 * alf) / (1.0 + 2.4 * n + 1.8 * alf);
        } else if (i == 2) {
            z = z + (15.0 + 6.25 * alf) / (1.0 + 0.9 * alf + 2.5 * n);
        } else {
            double ai = (double)(i - 2);
            z = z + ((1.0 + 2.55 * ai) / (1.9 * ai) + 1.26 * ai * alf / (1.0 + 3.5 * ai)) *
                        (z - x[i - 3]) / (1.0 + 0.3 * alf);
        }
        for (int its = 1; its <= maxit; ++its) {
            p1 = 1.0;
            p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                p3 = p2;
                p2 = p1;
                p1 = (((double)(2 * j - 1) + alf - z) * p2 - ((double)(j - 1) + alf) * p3) / (double)j;
            }
            pp = ((double)n * p1 - ((double)n + alf) * p2) / z;
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= eps) break;
        }
        x[i - 1] = z;
        /* exp(gammln(alf+n) - gammln(n)) is exactly 1 for alf = 0, the only
         * value rwaven uses; lgamma covers other alf. */
        double g = (alf == 0.0) ? 1.0 : exp(lgamma(alf + n) - lgamma((double)n));
        w[i - 1] = -g / (pp * (double)n * p2);
    }
}

/* src/rwaven.f90:49-151 */
int orc_rwaven(const orc_problem *p, int32_t *kwnanz, double *kwn, double *kwnwi,
               double *amin_out, double *amax_out)
{
    double amin = 1e9, amax = 0.0;
    double xke[4] = {0, 0, 0, 0}, yke[4] = {0, 0, 0, 0};
    for (int i = 0; i < p->nanz; ++i) {
        int elec[4];
        elec[0] = p->strnr[i] % 10000;
        elec[1] = (p->strnr[i] - elec[0]) / 10000;
        elec[2] = p->vnr[i] % 10000;
        elec[3] = (p->vnr[i] - elec[2]) / 10000;
        for (int j = 0; j < 4; ++j) {
            if (elec[j] > 0) {
                xke[j] = SX(p, p->enr[elec[j] - 1]);
                yke[j] = SY(p, p->enr[elec[j] - 1]);
            }
        }
        for (int v = 2; v < 4; ++v) {
            if (elec[v] <= 0) continue;
            for (int j = 0; j < 2; ++j) {
                if (elec[j] > 0) {
                    double x21 = xke[v] - xke[j], y21 = yke[v] - yke[j];
                    double dum = sqrt(x21 * x21 + y21 * y21);
                    amin = fmin(dum, amin);
                    amax = fmax(dum, amax);
                }
            }
        }
    }
    if (amin_out) *amin_out = amin;
    if (amax_out) *amax_out = amax;
    if (amin < 1e-12 || amax < 1e-12) return 73;
    const int lanz = 4;
    /* int(real(6d0*dlog10(amax/amin))): rounded to single precision first. */
    int ganz = (int)(float)(6.0 * log10(amax / amin));
    ganz = imax_i(ganz, 2);
    ganz = imin_i(ganz, 30 - lanz);
    *kwnanz = ganz + lanz;
    double kwn0 = 1.0 / (2.0 * amin);
    orc_gauleg(0.0, 1.0, kwn, kwnwi, ganz);
    for (int i = 0; i < ganz; ++i) {
        kwnwi[i] = 2.0 * kwn0 * kwnwi[i] * kwn[i];
        kwn[i] = kwn0 * kwn[i] * kwn[i];
    }
    orc_gaulag(kwn + ganz, kwnwi + ganz, lanz, 0.0);
    for (int i = ganz; i < ganz + lanz; ++i) {
        kwnwi[i] = kwn0 * kwnwi[i] * exp(kwn[i]);
        kwn[i] = kwn0 * (kwn[i] + 1.0);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Modified Bessel functions: src/bessi0.f90, bessi1.f90, bessk0.f90,
 * bessk1.f90 (the polynomial approximations of Abramowitz & Stegun
 * 9.8.1-9.8.8 as the reference writes them, with K0 = K1 = 0 for x > 500). */
static double orc_bessi0(double x)
{
    if (fabs(x) < 3.75) {
        double y = (x / 3.75) * (x / 3.75);
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 +
               y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))));
    }
    double ax = fabs(x), y = 3.75 / ax;
    return (exp(ax) / sqrt(ax)) * (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 +
           y * (-0.157565e-2 + y * (0.916281e-2 + y * (-0.2057706e-1 + y * (0.2635537e-1 +
           y * (-0.1647633e-1 + y * 0.392377e-2))))))));
}

static double orc_bessi1(double x)
{
    if (fabs(x) < 3.75) {
        double y = (x / 3.75) * (x / 3.75);
        return x * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 +
               y * (0.2658733e-1 + y * (0.301532e-2 + y * 0.32411e-3))))));
    }
    double ax = fabs(x), y = 3.75 / ax;
    return (exp(ax) / sqrt(ax)) * (0.39894228 + y * (-0.3988024e-1 + y * (-0.362018e-2 +
           y * (0.163801e-2 + y * (-0.1031555e-1 + y * (0.2282967e-1 + y * (-0.2895312e-1 +
           y * (0.1787654e-1 + y * -0.420059e-2))))))));
}

double orc_bessk0(double x)
{
    if (x <= 2.0) {
        double y = x * x / 4.0;
        return (-log(x / 2.0) * orc_bessi0(x)) + (-0.57721566 + y * (0.42278420 +
               y * (0.23069756 + y * (0.3488590e-1 + y * (0.262698e-2 + y * (0.10750e-3 +
               y * 0.74e-5))))));
    } else if (x > 5e2) {
        return 0.0;
    }
    double y = 2.0 / x;
    return (exp(-x) / sqrt(x)) * (1.25331414 + y * (-0.7832358e-1 + y * (0.2189568e-1 +
           y * (-0.1062446e-1 + y * (0.587872e-2 + y * (-0.251540e-2 + y * 0.53208e-3))))));
}

double orc_bessk1(double x)
{
    if (x <= 2.0) {
        double y = x * x / 4.0;
        return (log(x / 2.0) * orc_bessi1(x)) + (1.0 / x) * (1.0 + y * (0.15443144 +
               y * (-0.67278579 + y * (-0.18156897 + y * (-0.1919402e-1 + y * (-0.110404e-2 +
               y * -0.4686e-4))))));
    } else if (x > 5e2) {
        return 0.0;
    }
    double y = 2.0 / x;
    return (exp(-x) / sqrt(x)) * (1.25331414 + y * (0.23498619 + y * (-0.3655620e-1 +
           y * (0.1504268e-1 + y * (-0.780353e-2 + y * (0.325614e-2 + y * -0.68245e-3))))));
}

/* ------------------------------------------------------------------------ */
/* Element matrices.  src/elem1.f90:50-64, elem3.f90:62-94, elem5.f90:36-67,
 * elem8.f90:78-194.  mas/mam are row-major nk x nk (symmetric). */
static void orc_elem1(const double *xk, const double *yk, double *mam)
{
    static const int s4[2][2] = {{2, 1}, {1, 2}};
    double x21 = xk[1] - xk[0], y21 = yk[1] - yk[0];
    double l = sqrt(x21 * x21 + y21 * y21);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) mam[i * 2 + j] = l * (double)s4[i][j] / 6.0;
}

/* The three stencils of the linear triangle (stiffness split by the metric
 * coefficients a, b, c) and its consistent mass pattern. */
static const int tri_s1[3][3] = {{1, -1, 0}, {-1, 1, 0}, {0, 0, 0}};
static const int tri_s2[3][3] = {{2, -1, -1}, {-1, 0, 1}, {-1, 1, 0}};
static const int tri_s3[3][3] = {{1, 0, -1}, {0, 0, 0}, {-1, 0, 1}};
static const int tri_s4[3][3] = {{2, 1, 1}, {1, 2, 1}, {1, 1, 2}};

static int orc_elem3(const double *xk, const double *yk, double *mas, double *mam)
{
    double x21 = xk[1] - xk[0], x31 = xk[2] - xk[0];
    double y21 = yk[1] - yk[0], y31 = yk[2] - yk[0];
    double det = x21 * y31 - x31 * y21;
    if (det <= 0.0) return 26;
    double a = (x31 * x31 + y31 * y31) / det;
    double b = -(x31 * x21 + y31 * y21) / det;
    double c = (x21 * x21 + y21 * y21) / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            mas[i * 3 + j] = (a * tri_s1[i][j] + b * tri_s2[i][j] + c * tri_s3[i][j]) / 2.0;
            mam[i * 3 + j] = det * (double)tri_s4[i][j] / 2.4e1;
        }
    return 0;
}

static int orc_elem5(const double *xk, const double *yk, double *mas, double *mam)
{
    static const int s1[4][4] = {{2, -2, -1, 1}, {-2, 2, 1, -1}, {-1, 1, 2, -2}, {1, -1, -2, 2}};
    static const int s2[4][4] = {{1, 0, -1, 0}, {0, -1, 0, 1}, {-1, 0, 1, 0}, {0, 1, 0, -1}};
    static const int s3[4][4] = {{2, 1, -1, -2}, {1, 2, -2, -1}, {-1, -2, 2, 1}, {-2, -1, 1, 2}};
    static const int s4[4][4] = {{4, 2, 1, 2}, {2, 4, 2, 1}, {1, 2, 4, 2}, {2, 1, 2, 4}};
    double x21 = xk[1] - xk[0], x31 = xk[3] - xk[0];
    double y21 = yk[1] - yk[0], y31 = yk[3] - yk[0];
    double det = x21 * y31 - x31 * y21;
    if (det <= 0.0) return 26;
    double a = (x31 * x31 + y31 * y31) / det;
    double b = -(x31 * x21 + y31 * y21) / det;
    double c = (x21 * x21 + y21 * y21) / det;
    /* data statements fill column-major; the patterns are symmetric. */
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            mas[i * 4 + j] = (a * s1[j][i] + 3.0 * b * s2[j][i] + c * s3[j][i]) / 6.0;
            mam[i * 4 + j] = det * (double)s4[j][i] / 3.6e1;
        }
    return 0;
}

/* Quadrilateral as four triangles around the diagonal intersection, with
 * the centre node condensed out at wavenumber kwert (src/elem8.f90). */
static int orc_elem8(const double *xk, const double *yk, double kwert, double *kelmas)
{
    double xd[5], yd[5], mas[5][5], mam[5][5];
    memset(mas, 0, sizeof(mas));
    memset(mam, 0, sizeof(mam));
    double a1 = xk[2] - xk[0], a2 = xk[3] - xk[1];
    if (fabs(a1) <= 1e-12 || fabs(a2) <= 1e-12) return 26;
    a1 = (yk[2] - yk[0]) / a1;
    a2 = (yk[3] - yk[1]) / a2;
    if (fabs(a1 - a2) <= 1e-12) return 26;
    xd[4] = (a1 * xk[0] - yk[0] - a2 * xk[1] + yk[1]) / (a1 - a2);
    yd[4] = yk[0] + a1 * (xd[4] - xk[0]);
    for (int i = 0; i < 4; ++i) {
        xd[i] = xk[i];
        yd[i] = yk[i];
    }
    static const int sub[4][3] = {{0, 1, 4}, {1, 2, 4}, {4, 2, 3}, {0, 4, 3}};
    for (int t = 0; t < 4; ++t) {
        const int *ik = sub[t];
        double x21 = xd[ik[1]] - xd[ik[0]], x31 = xd[ik[2]] - xd[ik[0]];
        double y21 = yd[ik[1]] - yd[ik[0]], y31 = yd[ik[2]] - yd[ik[0]];
        double det = x21 * y31 - x31 * y21;
        if (det <= 1e-12) return 26;
        double a = (x31 * x31 + y31 * y31) / det;
        double b = -(x31 * x21 + y31 * y21) / det;
        double c = (x21 * x21 + y21 * y21) / det;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                mas[ik[i]][ik[j]] += (a * tri_s1[i][j] + b * tri_s2[i][j] + c * tri_s3[i][j]) / 2.0;
                mam[ik[i]][ik[j]] += det * (double)tri_s4[i][j] / 2.4e1;
            }
    }
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) mas[i][j] = mas[i][j] + kwert * kwert * mam[i][j];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) kelmas[i * 4 + j] = mas[i][j] - mas[i][4] * mas[4][j] / mas[4][4];
    return 0;
}

/* Mixed-boundary coefficient for a boundary segment (xk, yk) and source
 * electrode nelec at wavenumber ki: src/beta.f90:38-135. */
static int orc_beta(const orc_problem *p, const double *xk, const double *yk, double sytop,
                    int nelec, int ki, double *beta_out)
{
    double kw = p->kwn[ki - 1];
    double xs = SX(p, p->enr[nelec - 1]), ys = SY(p, p->enr[nelec - 1]);
    double xr = (xk[0] + xk[1]) / 2.0, yr = (yk[0] + yk[1]) / 2.0;
    double x3 = xr - xs;
    double y3m = (yr - sytop) - (ys - sytop);
    double y3p = (yr - sytop) + (ys - sytop);
    double r1m = sqrt(x3 * x3 + y3m * y3m);
    double r1p = sqrt(x3 * x3 + y3p * y3p);
    double x4 = yk[0] - yk[1], y4 = xk[1] - xk[0];
    double r2 = sqrt(x4 * x4 + y4 * y4);
    if (r1m < 1e-12 || r1p < 1e-12 || r2 < 1e-12) return 35;
    double cthetm = (x3 * x4 + y3m * y4) / r1m / r2;
    double cthetp = (x3 * x4 + y3p * y4) / r1p / r2;
    double bk0m = orc_bessk0(r1m * kw), bk0p = orc_bessk0(r1p * kw);
    double bk1m = orc_bessk1(r1m * kw), bk1p = orc_bessk1(r1p * kw);
    double beta;
    if (bk0m + bk0p == 0.0)
        beta = (cthetm + cthetp) / 2.0;
    else
        beta = (cthetm * bk1m + cthetp * bk1p) / (bk0m + bk0p);
    *beta_out = kw * beta;
    return 0;
}

/* src/bsytop.f90:35-69: running mean of the type-12 segment midpoint depths */
static double orc_bsytop(const orc_problem *p)
{
    double sytop = 0.0;
    int iel = 0;
    for (int i = 0; i < p->typanz; ++i) {
        if (p->typ[i] == 12) {
            int nkel = p->selanz[i];
            sytop = 0.0;
            for (int j = 1; j <= p->nelanz[i]; ++j) {
                ++iel;
                double sp = 0.0;
                for (int ik = 1; ik <= nkel; ++ik) sp += SY(p, NREL(p, iel, ik));
                sp = sp / (double)nkel;
                if (j == 1)
                    sytop = sp;
                else
                    sytop = (sytop * (double)(j - 1) + sp) / (double)j;
            }
        } else {
            iel += p->nelanz[i];
        }
    }
    return sytop;
}

/* src/precal.f90:57-208 */
int orc_precal(const orc_problem *p, int lsytop, double *elbg, double *relbg, double *kg,
               int32_t *lbeta_out, int32_t *lrandb_out)
{
    int lbeta = 0, lrandb = 0;
    int iel = 0;
    const int nmn = NMN(p);
    const int ne_tot = p->elanz + p->relanz;
    double sytop = lsytop ? orc_bsytop(p) : 0.0;
    double xk[8], yk[8], mas[64], mam[64];
    for (int i = 0; i < p->typanz; ++i) {
        int ntyp = p->typ[i], nkel = p->selanz[i];
        for (int j = 0; j < p->nelanz[i]; ++j) {
            ++iel;
            for (int m = 1; m <= nkel; ++m) {
                int node = p->nrel[(size_t)(m - 1) * ne_tot + iel - 1];
                xk[m - 1] = SX(p, node);
                yk[m - 1] = SY(p, node);
            }
            if (ntyp == 11) {
                if (lrandb) return 101;
                lbeta = 1;
                orc_elem1(xk, yk, mam);
                int rel = iel - p->elanz;
                if (rel <= 0) return 36;
                int imn = 0;
                for (int m = 0; m < nkel; ++m)
                    for (int n = 0; n <= m; ++n) {
                        ++imn;
                        relbg[(size_t)(imn - 1) * p->relanz + rel - 1] = mam[m * 2 + n];
                    }
                for (int l = 1; l <= p->eanz; ++l)
                    for (int k = 1; k <= p->kwnanz; ++k) {
                        double b;
                        int e = orc_beta(p, xk, yk, sytop, l, k, &b);
                        if (e) return e;
                        kg[(((size_t)k - 1) * p->eanz + l - 1) * p->relanz + rel - 1] = b;
                    }
            } else if (ntyp == 12) {
                continue;
            } else if (ntyp == 13) {
                if (lbeta) return 101;
                lrandb = 1;
                continue;
            } else if (ntyp == 8) {
                for (int k = 1; k <= p->kwnanz; ++k) {
                    int e = orc_elem8(xk, yk, p->kwn[k - 1], mas);
                    if (e) return e;
                    int imn = 0;
                    for (int m = 0; m < nkel; ++m)
                        for (int n = 0; n <= m; ++n) {
                            ++imn;
                            elbg[(((size_t)k - 1) * nmn + imn - 1) * p->elanz + iel - 1] = mas[m * 4 + n];
                        }
                }
            } else {
                int e;
                if (ntyp == 3)
                    e = orc_elem3(xk, yk, mas, mam);
                else if (ntyp == 5)
                    e = orc_elem5(xk, yk, mas, mam);
                else
                    return 18;
                if (e) return e;
                for (int k = 1; k <= p->kwnanz; ++k) {
                    int imn = 0;
                    double kk = p->kwn[k - 1];
                    for (int m = 0; m < nkel; ++m)
                        for (int n = 0; n <= m; ++n) {
                            ++imn;
                            elbg[(((size_t)k - 1) * nmn + imn - 1) * p->elanz + iel - 1] =
                                mas[m * nkel + n] + mam[m * nkel + n] * kk * kk;
                        }
                }
            }
        }
    }
    if (lbeta_out) *lbeta_out = lbeta;
    if (lrandb_out) *lrandb_out = lrandb;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Assembly: src/kompab.f90:75-183 (complex) and src/kompadc.f90:72-165
 * (real).  Band a((mb+1)*sanz): entry (m, n), m >= n, at a(m*mb + n). */
int orc_kompab(const orc_problem *p, int nelec, int ki, const dcplx *sigma, dcplx *a, dcplx *b)
{
    const int mb = p->mb, sanz = p->sanz;
    memset(a, 0, sizeof(dcplx) * (size_t)(mb + 1) * sanz);
    memset(b, 0, sizeof(dcplx) * (size_t)sanz);
    int iel = 0;
    for (int i = 0; i < p->typanz; ++i) {
        int ntyp = p->typ[i], nkel = p->selanz[i];
        for (int j = 0; j < p->nelanz[i]; ++j) {
            ++iel;
            int ikl = 0;
            if (ntyp > 11) continue;
            for (int k = 1; k <= nkel; ++k) {
                int nzp = NREL(p, iel, k);
                for (int l = 1; l <= k; ++l) {
                    int nnp = NREL(p, iel, l);
                    int idif = abs(nzp - nnp);
                    if (idif > mb) return 19;
                    ++ikl;
                    int im = imax_i(nzp, nnp) * mb + imin_i(nzp, nnp);
                    double dum;
                    dcplx dum2;
                    if (ntyp == 11) {
                        int rel = iel - p->elanz;
                        dum = RELBG(p, rel, ikl) * KG(p, rel, nelec, ki);
                        dum2 = sigma[p->rnr[rel - 1] - 1];
                    } else {
                        dum = ELBG(p, iel, ikl, ki);
                        dum2 = sigma[iel - 1];
                    }
                    a[im - 1] = a[im - 1] + dum * dum2;
                }
            }
        }
    }
    b[p->enr[nelec - 1] - 1] = -1.0;
    if (p->lsink) b[p->nsink - 1] = 1.0;
    return 0;
}

static int orc_kompadc(const orc_problem *p, int nelec, int ki, const dcplx *sigma, double *a,
                       double *b)
{
    const int mb = p->mb, sanz = p->sanz;
    memset(a, 0, sizeof(double) * (size_t)(mb + 1) * sanz);
    memset(b, 0, sizeof(double) * (size_t)sanz);
    int iel = 0;
    for (int i = 0; i < p->typanz; ++i) {
        int ntyp = p->typ[i], nkel = p->selanz[i];
        for (int j = 0; j < p->nelanz[i]; ++j) {
            ++iel;
            int ikl = 0;
            if (ntyp > 11) continue;
            for (int k = 1; k <= nkel; ++k) {
                int nzp = NREL(p, iel, k);
                for (int l = 1; l <= k; ++l) {
                    int nnp = NREL(p, iel, l);
                    if (abs(nzp - nnp) > mb) return 19;
                    ++ikl;
                    int im = imax_i(nzp, nnp) * mb + imin_i(nzp, nnp);
                    double dum, dum2;
                    if (ntyp == 11) {
                        int rel = iel - p->elanz;
                        dum = RELBG(p, rel, ikl) * KG(p, rel, nelec, ki);
                        dum2 = creal(sigma[p->rnr[rel - 1] - 1]);
                    } else {
                        dum = ELBG(p, iel, ikl, ki);
                        dum2 = creal(sigma[iel - 1]);
                    }
                    a[im - 1] = a[im - 1] + dum * dum2;
                }
            }
        }
    }
    b[p->enr[nelec - 1] - 1] = -1.0;
    if (p->lsink) b[p->nsink - 1] = 1.0;
    return 0;
}

/* Dirichlet nodes of element type 13: src/randb.f90:40-82 (randdc.f90 is
 * the real twin).  Generic over the element type via a macro. */
#define RANDB_BODY(ZERO, ONE)                                                   \
    const int mb = p->mb, sanz = p->sanz, m1 = mb + 1;                          \
    int iel = 0;                                                                \
    for (int i2 = 0; i2 < p->typanz; ++i2) {                                    \
        int ntyp = p->typ[i2], nkel = p->selanz[i2];                            \
        for (int j2 = 0; j2 < p->nelanz[i2]; ++j2) {                            \
            ++iel;                                                              \
            if (ntyp != 13) continue;                                           \
            for (int ir = 1; ir <= nkel; ++ir) {                                \
                int k = NREL(p, iel, ir);                                       \
                b[k - 1] = ZERO;                                                \
                int idk = k * m1;                                               \
                a[idk - 1] = ONE;                                               \
                if (k != 1) {                                                   \
                    for (int i = imax_i(1, mb + 2 - k); i <= mb; ++i)           \
                        a[idk + i - m1 - 1] = ZERO;                             \
                }                                                               \
                if (k == sanz) continue;                                        \
                for (int i = imax_i(1, k - sanz + m1); i <= mb; ++i) {          \
                    int j = k - i + m1;                                         \
                    a[(j - 1) * m1 + i - 1] = ZERO;                             \
                }                                                               \
            }                                                                   \
        }                                                                       \
    }

static void orc_randb(const orc_problem *p, dcplx *a, dcplx *b) { RANDB_BODY(0.0, 1.0) }
static void orc_randdc(const orc_problem *p, double *a, double *b) { RANDB_BODY(0.0, 1.0) }

/* Prescribed boundary values (boundary.dat): src/randb2.f90:39-79 and
 * src/randbdc2.f90 (real twin, real parts of the values). */
#define RANDB2_BODY(T, VAL)                                                      \
    const int mb = p->mb, sanz = p->sanz, m1 = mb + 1;                           \
    for (int ir = 0; ir < p->rwdanz; ++ir) {                                     \
        int k = p->rwdnr[ir];                                                    \
        T rwert = VAL(p->rwd[ir]);                                               \
        b[k - 1] = -rwert;                                                       \
        int idk = k * m1;                                                        \
        a[idk - 1] = 1.0;                                                        \
        if (k != 1) {                                                            \
            for (int i = imax_i(1, mb + 2 - k); i <= mb; ++i) {                  \
                int j = k + i - m1, ki = idk + i - m1;                           \
                b[j - 1] = b[j - 1] + rwert * a[ki - 1];                         \
                a[ki - 1] = 0.0;                                                 \
            }                                                                    \
        }                                                                        \
        if (k == sanz) continue;                                                 \
        for (int i = imax_i(1, k - sanz + m1); i <= mb; ++i) {                   \
            int j = k - i + m1, ji = (j - 1) * m1 + i;                           \
            b[j - 1] = b[j - 1] + rwert * a[ji - 1];                             \
            a[ji - 1] = 0.0;                                                     \
        }                                                                        \
    }

#define ID_C(x) (x)
static void orc_randb2(const orc_problem *p, dcplx *a, dcplx *b) { RANDB2_BODY(dcplx, ID_C) }
static void orc_randbdc2(const orc_problem *p, double *a, double *b) { RANDB2_BODY(double, creal) }

/* src/scalab.f90:52-76 */
int orc_scalab(const orc_problem *p, dcplx *a, dcplx *b, double *fak)
{
    const int mb = p->mb, sanz = p->sanz;
    for (int i = 1; i <= sanz; ++i) {
        int idi = i * (mb + 1);
        double dum = cabs(a[idi - 1]);
        if (dum <= 0.0) return 27;
        a[idi - 1] = a[idi - 1] / dum;
        fak[i - 1] = 1.0 / sqrt(dum);
        b[i - 1] = b[i - 1] * fak[i - 1];
        if (i == 1) continue;
        int i0 = i * mb, ja = imax_i(1, i - mb);
        for (int j = ja; j <= i - 1; ++j) a[i0 + j - 1] = a[i0 + j - 1] * (fak[i - 1] * fak[j - 1]);
    }
    return 0;
}

/* src/scaldc.f90:49-73 */
static int orc_scaldc(const orc_problem *p, double *a, double *b, double *fak)
{
    const int mb = p->mb, sanz = p->sanz;
    for (int i = 1; i <= sanz; ++i) {
        int idi = i * (mb + 1);
        double dum = a[idi - 1];
        if (dum <= 0.0) return 27;
        a[idi - 1] = 1.0;
        fak[i - 1] = 1.0 / sqrt(dum);
        b[i - 1] = b[i - 1] * fak[i - 1];
        if (i == 1) continue;
        int i0 = i * mb, ja = imax_i(1, i - mb);
        for (int j = ja; j <= i - 1; ++j) a[i0 + j - 1] = a[i0 + j - 1] * fak[i - 1] * fak[j - 1];
    }
    return 0;
}

/* Row-oriented band Cholesky, complex symmetric without conjugation:
 * src/chol.f90:44-78 (choldc.f90:42-78 is the real twin). */
int orc_chol(const orc_problem *p, dcplx *a)
{
    const int mb = p->mb, m1 = mb + 1;
    for (int i = 1; i <= p->sanz; ++i) {
        int idi = i * m1, fi = imax_i(1, i - mb), i0 = idi - i;
        for (int j = fi; j <= i; ++j) {
            int ij = i0 + j, j0 = j * mb;
            dcplx s = a[ij - 1];
            for (int k = fi; k <= j - 1; ++k) s = s - a[i0 + k - 1] * a[j0 + k - 1];
            if (j < i) {
                a[ij - 1] = s / a[j * m1 - 1];
            } else {
                if (cabs(s) <= 0.0) return 28;
                a[idi - 1] = csqrt(s);
            }
        }
    }
    return 0;
}

static int orc_choldc(const orc_problem *p, double *a)
{
    const int mb = p->mb, m1 = mb + 1;
    for (int i = 1; i <= p->sanz; ++i) {
        int idi = i * m1, fi = imax_i(1, i - mb), i0 = idi - i;
        for (int j = fi; j <= i; ++j) {
            int ij = i0 + j, j0 = j * mb;
            double s = a[ij - 1];
            for (int k = fi; k <= j - 1; ++k) s = s - a[i0 + k - 1] * a[j0 + k - 1];
            if (j < i) {
                a[ij - 1] = s / a[j * m1 - 1];
            } else {
                if (s <= 0.0) return 28;
                a[idi - 1] = sqrt(s);
            }
        }
    }
    return 0;
}

/* Forward / back substitution for A x + b = 0: src/vre.f90:43-69
 * (vredc.f90:47-77 real twin).  The back substitution reuses idi from the
 * end of the forward sweep, as the reference does. */
void orc_vre(const orc_problem *p, const dcplx *a, const dcplx *b, dcplx *pot)
{
    const int mb = p->mb, m1 = mb + 1, sanz = p->sanz;
    int idi = 0;
    for (int i = 1; i <= sanz; ++i) {
        idi = i * m1;
        dcplx s = b[i - 1];
        int i0 = idi - i, jlow = imax_i(1, i - mb);
        for (int j = jlow; j <= i - 1; ++j) s = s - a[i0 + j - 1] * pot[j - 1];
        pot[i - 1] = s / a[idi - 1];
    }
    for (int i = sanz; i >= 1; --i) {
        pot[i - 1] = -pot[i - 1] / a[idi - 1];
        int jlow = imax_i(1, i - mb), i0 = idi - i;
        for (int j = jlow; j <= i - 1; ++j) pot[j - 1] = pot[j - 1] + a[i0 + j - 1] * pot[i - 1];
        idi = idi - m1;
    }
}

static void orc_vredc(const orc_problem *p, const double *a, const double *b, double *pot)
{
    const int mb = p->mb, m1 = mb + 1, sanz = p->sanz;
    int idi = 0;
    for (int i = 1; i <= sanz; ++i) {
        idi = i * m1;
        double s = b[i - 1];
        int i0 = idi - i, jlow = imax_i(1, i - mb);
        for (int j = jlow; j <= i - 1; ++j) s = s - a[i0 + j - 1] * pot[j - 1];
        pot[i - 1] = s / a[idi - 1];
    }
    for (int i = sanz; i >= 1; --i) {
        pot[i - 1] = -pot[i - 1] / a[idi - 1];
        int jlow = imax_i(1, i - mb), i0 = idi - i;
        for (int j = jlow; j <= i - 1; ++j) pot[j - 1] = pot[j - 1] + a[i0 + j - 1] * pot[i - 1];
        idi = idi - m1;
    }
}

/* ------------------------------------------------------------------------ */
/* The wavenumber x electrode loop: src/inv.f90:343-414 (DC) and :426-484
 * (complex); src/fem.f90:328-397 is the CRMod copy.  OpenMP over k. */
int orc_forward(const orc_problem *p, const dcplx *sigma, int ldc, int nthreads, dcplx *kpot)
{
    const int sanz = p->sanz, mb = p->mb;
    int *kerr = (int *)calloc((size_t)p->kwnanz + 1, sizeof(int));
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
#endif
    for (int k = 1; k <= p->kwnanz; ++k) {
        int err = 0;
        size_t band = (size_t)(mb + 1) * sanz;
        double *fak = (double *)malloc(sizeof(double) * sanz);
        if (ldc) {
            double *a = (double *)malloc(sizeof(double) * band);
            double *b = (double *)malloc(sizeof(double) * sanz);
            double *pot = (double *)malloc(sizeof(double) * sanz);
            for (int l = 1; l <= p->eanz && !err; ++l) {
                int e = 0;
                if (p->lbeta || l == 1) {
                    e = orc_kompadc(p, l, k, sigma, a, b);
                    if (!e && p->lrandb) orc_randdc(p, a, b);
                    if (!e && p->lrandb2) orc_randbdc2(p, a, b);
                    if (!e) e = orc_scaldc(p, a, b, fak);
                    if (!e) e = orc_choldc(p, a);
                } else {
                    /* src/kompbdc.f90 */
                    memset(b, 0, sizeof(double) * sanz);
                    b[p->enr[l - 1] - 1] = -fak[p->enr[l - 1] - 1];
                    if (p->lsink) b[p->nsink - 1] = fak[p->nsink - 1];
                }
                if (e) {
                    err = e;
                    break;
                }
                orc_vredc(p, a, b, pot);
                for (int j = 1; j <= sanz; ++j) KPOT(p, kpot, j, l, k) = pot[j - 1] * fak[j - 1];
            }
            free(a);
            free(b);
            free(pot);
        } else {
            dcplx *a = (dcplx *)malloc(sizeof(dcplx) * band);
            dcplx *b = (dcplx *)malloc(sizeof(dcplx) * sanz);
            dcplx *pot = (dcplx *)malloc(sizeof(dcplx) * sanz);
            for (int l = 1; l <= p->eanz && !err; ++l) {
                int e = 0;
                if (p->lbeta || l == 1) {
                    e = orc_kompab(p, l, k, sigma, a, b);
                    if (!e && p->lrandb) orc_randb(p, a, b);
                    if (!e && p->lrandb2) orc_randb2(p, a, b);
                    if (!e) e = orc_scalab(p, a, b, fak);
                    if (!e) e = orc_chol(p, a);
                } else {
                    /* src/kompb.f90:39-66 */
                    memset(b, 0, sizeof(dcplx) * sanz);
                    b[p->enr[l - 1] - 1] = -fak[p->enr[l - 1] - 1];
                    if (p->lsink) b[p->nsink - 1] = fak[p->nsink - 1];
                }
                if (e) {
                    err = e;
                    break;
                }
                orc_vre(p, a, b, pot);
                for (int j = 1; j <= sanz; ++j) KPOT(p, kpot, j, l, k) = pot[j - 1] * fak[j - 1];
            }
            free(a);
            free(b);
            free(pot);
        }
        free(fak);
        kerr[k] = err;
    }
    int err = 0;
    for (int k = 1; k <= p->kwnanz && !err; ++k) err = kerr[k];
    free(kerr);
    return err;
}

/* src/rtrafo.f90:46-90 (swrtr = 0: hpot = kpot(:,:,1)) */
void orc_rtrafo(const orc_problem *p, const dcplx *kpot, dcplx *hpot)
{
    const double pi = acos(-1.0);
    for (int l = 1; l <= p->eanz; ++l)
        for (int j = 1; j <= p->sanz; ++j) {
            dcplx s = 0.0;
            if (p->swrtr == 0) {
                s = KPOT(p, kpot, j, l, 1);
            } else {
                for (int k = 1; k <= p->kwnanz; ++k) s = s + KPOT(p, kpot, j, l, k) * p->kwnwi[k - 1];
                s = s / pi;
            }
            hpot[(size_t)(l - 1) * p->sanz + j - 1] = s;
        }
}

static inline void decode4(int32_t strnr, int32_t vnr, int *e)
{
    e[0] = strnr % 10000;
    e[1] = (strnr - e[0]) / 10000;
    e[2] = vnr % 10000;
    e[3] = (vnr - e[2]) / 10000;
}

/* Four-pole superposition shared by bvolti / bvolt. */
static dcplx orc_superpose(const orc_problem *p, const dcplx *hpot, const int *e)
{
#define HP(node, l) hpot[(size_t)((l) - 1) * p->sanz + (node) - 1]
#define TERM(ep, ec) \
    ((double)(imin_i(ep, 1) * imin_i(ec, 1)) * HP(p->enr[imax_i(ep, 1) - 1], imax_i(ec, 1)))
    dcplx d1 = TERM(e[3], e[1]);
    dcplx d2 = TERM(e[3], e[0]);
    dcplx d3 = TERM(e[2], e[1]);
    dcplx d4 = TERM(e[2], e[0]);
    return (d1 - d2) - (d3 - d4);
#undef TERM
#undef HP
}

/* src/bvolti.f90:43-89 */
int orc_bvolti(const orc_problem *p, const dcplx *hpot, dcplx *volt, dcplx *sigmaa)
{
    for (int i = 0; i < p->nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        volt[i] = orc_superpose(p, hpot, e);
        if (cabs(volt[i]) == 0.0) return 82;
        sigmaa[i] = -clog(volt[i]);
    }
    return 0;
}

/* src/bvolt.f90:40-79 */
void orc_bvolt(const orc_problem *p, const dcplx *hpot, const double *kfak, dcplx *volt,
               dcplx *sigmaa)
{
    for (int i = 0; i < p->nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        volt[i] = orc_superpose(p, hpot, e);
        sigmaa[i] = (kfak ? kfak[i] : 1.0) * volt[i];
    }
}

/* src/bkfak.f90:46-136 */
int orc_bkfak(const orc_problem *p, double *kfak)
{
    const double pi = acos(-1.0);
    double xk[4] = {0, 0, 0, 0}, yk[4] = {0, 0, 0, 0};
    for (int i = 0; i < p->nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        for (int q = 0; q < 4; ++q)
            if (e[q] > 0) {
                xk[q] = SX(p, p->enr[e[q] - 1]);
                yk[q] = SY(p, p->enr[e[q] - 1]);
            }
        double r[4];
        /* r4: (3,1), r3: (3,2), r2: (4,1), r1: (4,2) */
        static const int pr[4][2] = {{3, 1}, {3, 0}, {2, 1}, {2, 0}};
        for (int q = 0; q < 4; ++q) {
            int u = pr[q][0], v = pr[q][1];
            if (e[u] > 0 && e[v] > 0) {
                double dx = xk[u] - xk[v], dym = yk[u] - yk[v], dyp = yk[u] + yk[v];
                dym = 1.0 / sqrt(dx * dx + dym * dym);
                dyp = 1.0 / sqrt(dx * dx + dyp * dyp);
                r[q] = dym + dyp;
            } else {
                r[q] = 0.0;
            }
        }
        /* r[0]=r1, r[1]=r2, r[2]=r3, r[3]=r4 */
        double dum = (r[0] - r[1]) - (r[2] - r[3]);
        if (fabs(dum) == 0.0) return 93;
        kfak[i] = 4.0 * pi / dum;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Reciprocity sensitivities.  hsens(k) = sum_{mi,mj} elbg(iel,imn,k) *
 * (phi_C2 - phi_C1)(nrel(iel,mj)) * (phi_P2 - phi_P1)(nrel(iel,mi)). */
static inline dcplx orc_hsens_elem(const orc_problem *p, const dcplx *kpot, int iel, int nkel,
                                   int k, const int *e)
{
    dcplx sup[4] = {0, 0, 0, 0}, h = 0.0;
    for (int mi = 1; mi <= nkel; ++mi) {
        int nzp = NREL(p, iel, mi);
        for (int mj = 1; mj <= nkel; ++mj) {
            int nnp = NREL(p, iel, mj);
            int imx = imax_i(mi, mj), imn_ = imin_i(mi, mj);
            int imn = imx * (imx - 1) / 2 + imn_;
            if (e[0] > 0) sup[0] = KPOT(p, kpot, nnp, e[0], k);
            if (e[1] > 0) sup[1] = KPOT(p, kpot, nnp, e[1], k);
            if (e[2] > 0) sup[2] = KPOT(p, kpot, nzp, e[2], k);
            if (e[3] > 0) sup[3] = KPOT(p, kpot, nzp, e[3], k);
            dcplx dum = (sup[1] - sup[0]) * (sup[3] - sup[2]);
            h = h + ELBG(p, iel, imn, k) * dum;
        }
    }
    return h;
}

/* src/bsensi.f90:82-188 */
void orc_bsensi(const orc_problem *p, const dcplx *kpot, const dcplx *sigma, const dcplx *volt,
                int nthreads, dcplx *sens)
{
    const double pi = acos(-1.0);
    const int nanz = p->nanz;
    memset(sens, 0, sizeof(dcplx) * (size_t)nanz * p->elanz);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(guided, 256) num_threads(nthreads)
#endif
    for (int i = 0; i < nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        int iel = 0;
        for (int ity = 0; ity < p->typanz; ++ity) {
            int ntyp = p->typ[ity], nkel = p->selanz[ity];
            if (ntyp > 10) continue;
            for (int jn = 0; jn < p->nelanz[ity]; ++jn) {
                ++iel;
                dcplx dum;
                if (p->swrtr == 0) {
                    dum = orc_hsens_elem(p, kpot, iel, nkel, 1, e);
                } else {
                    dum = 0.0;
                    for (int k = 1; k <= p->kwnanz; ++k)
                        dum = dum + orc_hsens_elem(p, kpot, iel, nkel, k, e) * p->kwnwi[k - 1];
                    dum = dum / pi;
                }
                size_t idx = (size_t)(iel - 1) * nanz + i;
                sens[idx] = sens[idx] + dum * sigma[iel - 1] / volt[i];
            }
        }
    }
}

/* src/bsendc.f90:62-179 (uses the real parts of kpot) */
void orc_bsendc(const orc_problem *p, const dcplx *kpot, const dcplx *sigma, const dcplx *volt,
                int nthreads, double *sensdc)
{
    const double pi = acos(-1.0);
    const int nanz = p->nanz;
    memset(sensdc, 0, sizeof(double) * (size_t)nanz * p->elanz);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(guided, 256) num_threads(nthreads)
#endif
    for (int i = 0; i < nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        int iel = 0;
        for (int ity = 0; ity < p->typanz; ++ity) {
            int ntyp = p->typ[ity], nkel = p->selanz[ity];
            if (ntyp > 10) continue;
            for (int jn = 0; jn < p->nelanz[ity]; ++jn) {
                ++iel;
                double dum = 0.0;
                int kmax = (p->swrtr == 0) ? 1 : p->kwnanz;
                for (int k = 1; k <= kmax; ++k) {
                    double sup[4] = {0, 0, 0, 0}, h = 0.0;
                    for (int mi = 1; mi <= nkel; ++mi) {
                        int nzp = NREL(p, iel, mi);
                        for (int mj = 1; mj <= nkel; ++mj) {
                            int nnp = NREL(p, iel, mj);
                            int imx = imax_i(mi, mj), imn_ = imin_i(mi, mj);
                            int imn = imx * (imx - 1) / 2 + imn_;
                            if (e[0] > 0) sup[0] = creal(KPOT(p, kpot, nnp, e[0], k));
                            if (e[1] > 0) sup[1] = creal(KPOT(p, kpot, nnp, e[1], k));
                            if (e[2] > 0) sup[2] = creal(KPOT(p, kpot, nzp, e[2], k));
                            if (e[3] > 0) sup[3] = creal(KPOT(p, kpot, nzp, e[3], k));
                            h = h + ELBG(p, iel, imn, k) * ((sup[1] - sup[0]) * (sup[3] - sup[2]));
                        }
                    }
                    if (p->swrtr == 0)
                        dum = h;
                    else
                        dum = dum + h * p->kwnwi[k - 1];
                }
                if (p->swrtr != 0) dum = dum / pi;
                size_t idx = (size_t)(iel - 1) * nanz + i;
                sensdc[idx] = sensdc[idx] + dum * creal(sigma[iel - 1] / volt[i]);
            }
        }
    }
}

/* src/bsens.f90:82-193 (CRMod raw sensitivities) */
void orc_bsens(const orc_problem *p, const dcplx *kpot, const double *strom, int nthreads,
               dcplx *sens)
{
    const double pi = acos(-1.0);
    const int nanz = p->nanz;
    memset(sens, 0, sizeof(dcplx) * (size_t)nanz * p->elanz);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(guided, 256) num_threads(nthreads)
#endif
    for (int i = 0; i < nanz; ++i) {
        int e[4];
        decode4(p->strnr[i], p->vnr[i], e);
        double st = strom ? strom[i] : 1.0;
        int iel = 0;
        for (int ity = 0; ity < p->typanz; ++ity) {
            int ntyp = p->typ[ity], nkel = p->selanz[ity];
            if (ntyp > 10) continue;
            for (int jn = 0; jn < p->nelanz[ity]; ++jn) {
                ++iel;
                dcplx dum;
                if (p->swrtr == 0) {
                    dum = orc_hsens_elem(p, kpot, iel, nkel, 1, e) * st;
                } else {
                    dum = 0.0;
                    for (int k = 1; k <= p->kwnanz; ++k)
                        dum = dum + orc_hsens_elem(p, kpot, iel, nkel, k, e) * p->kwnwi[k - 1];
                    dum = dum * (st / pi);
                }
                size_t idx = (size_t)(iel - 1) * nanz + i;
                sens[idx] = sens[idx] - dum;
            }
        }
    }
}

/* src/refsig.f90:7-73 */
dcplx orc_refsig(const orc_problem *p, const dcplx *sigma)
{
    double area = 0.0;
    dcplx s0 = 0.0;
    int iel = 0;
    for (int i = 0; i < p->typanz; ++i)
        for (int j = 0; j < p->nelanz[i]; ++j) {
            ++iel;
            if (p->typ[i] > 10) continue;
            double xk = SX(p, NREL(p, iel, 1)), yk = SY(p, NREL(p, iel, 1));
            double ax = SX(p, NREL(p, iel, 2)) - xk, ay = SY(p, NREL(p, iel, 2)) - yk;
            double bx = SX(p, NREL(p, iel, 3)) - xk, by = SY(p, NREL(p, iel, 3)) - yk;
            double dum = 0.0;
            if (p->typ[i] == 3) {
                dum = fabs(ax * by - ay * bx) / 2.0;
            } else if (p->typ[i] == 5 || p->typ[i] == 8) {
                double cx = SX(p, NREL(p, iel, 4)) - xk, cy = SY(p, NREL(p, iel, 4)) - yk;
                dum = (fabs(ax * by - ay * bx) + fabs(bx * cy - by * cx)) / 2.0;
            }
            s0 = s0 + dum * clog(sigma[iel - 1]);
            area = area + dum;
        }
    return cexp(s0 / area);
}

/* ------------------------------------------------------------------------ */
/* Neighbour table: src/bnachbar.f90:52-90 (element i and j share the edge
 * (ik, ik+1 mod n) in either orientation). */
void orc_bnachbar(const orc_problem *p, int32_t *nachbar)
{
    const int n = p->maxnodes, E = p->elanz;
    memset(nachbar, 0, sizeof(int32_t) * (size_t)E * (n + 1));
    for (int i = 1; i <= E; ++i)
        for (int ik = 1; ik <= n; ++ik) {
            int ik1 = NREL(p, i, ik), ik2 = NREL(p, i, ik % n + 1);
            for (int j = 1; j <= E; ++j) {
                if (j == i) continue;
                for (int jk = 1; jk <= n; ++jk) {
                    int jk1 = NREL(p, j, jk), jk2 = NREL(p, j, jk % n + 1);
                    if ((ik1 == jk1 && ik2 == jk2) || (ik1 == jk2 && ik2 == jk1)) {
                        nachbar[(size_t)(ik - 1) * E + i - 1] = j;
                        nachbar[(size_t)n * E + i - 1] += 1;
                    }
                }
            }
        }
}

/* Element midpoints espx/espy as set in src/relem.f90 */
void orc_esp(const orc_problem *p, double *espx, double *espy)
{
    int iel = 0, ifln = 0;
    for (int i = 0; i < p->typanz; ++i)
        for (int j = 0; j < p->nelanz[i]; ++j) {
            ++iel;
            if (p->typ[i] >= 10) continue;
            double sx = 0.0, sy = 0.0;
            for (int k = 1; k <= p->selanz[i]; ++k) {
                sx += SX(p, NREL(p, iel, k));
                sy += SY(p, NREL(p, iel, k));
            }
            espx[ifln] = sx / p->selanz[i];
            espy[ifln] = sy / p->selanz[i];
            ++ifln;
        }
}

/* src/bsmatm_mod.f90:364-460 (bsmatmtri, no decouplings) */
void orc_bsmatmtri(const orc_problem *p, const int32_t *nachbar, const double *espx,
                   const double *espy, double alfx, double alfz, double *smatm)
{
    const int n = p->maxnodes, E = p->elanz;
    memset(smatm, 0, sizeof(double) * (size_t)E * (n + 1));
    for (int i = 1; i <= E; ++i) {
        double sp1x = espx[i - 1], sp1y = espy[i - 1];
        for (int k = 1; k <= n; ++k) {
            int nxt = k % n + 1;
            double dx = SX(p, NREL(p, i, k)) - SX(p, NREL(p, i, nxt));
            double dy = SY(p, NREL(p, i, k)) - SY(p, NREL(p, i, nxt));
            double edglen = sqrt(dx * dx + dy * dy);
            int nb = nachbar[(size_t)(k - 1) * E + i - 1];
            if (nb > 0) {
                double sp2x = espx[nb - 1], sp2y = espy[nb - 1];
                double ddx = sp1x - sp2x, ddy = sp1y - sp2y;
                double dist = sqrt(ddx * ddx + ddy * ddy);
                double ang = atan2(ddy, ddx);
                double cx = alfx * cos(ang), sz = alfz * sin(ang);
                double alfgeo = sqrt(cx * cx + sz * sz);
                double rs = edglen / dist * alfgeo;
                smatm[(size_t)(k - 1) * E + i - 1] = -rs;
                smatm[(size_t)n * E + i - 1] += rs;
            }
        }
    }
}

/* src/bsmatm_mod.f90:190-362 (bsmatmreg, no discontinuities) */
void orc_bsmatmreg(const orc_problem *p, int nx, int nz, double alfx, double alfz, double *smatm)
{
    const int manz = nx * nz;
#define KX(i, j) (((i) - 1) * nx + (j))
#define SM(m, c) smatm[(size_t)((c) - 1) * manz + (m) - 1]
    memset(smatm, 0, sizeof(double) * (size_t)manz * 3);
    for (int i = 1; i <= nz; ++i)
        for (int j = 1; j <= nx; ++j) {
            int e = KX(i, j);
            double dzleft = fabs(SY(p, NREL(p, e, 4)) - SY(p, NREL(p, e, 1)));
            double dzright = fabs(SY(p, NREL(p, e, 3)) - SY(p, NREL(p, e, 2)));
            double xmean = 0.0;
            for (int l = 1; l <= 4; ++l) xmean += SX(p, NREL(p, e, l));
            xmean /= 4.0;
            if (j > 1) {
                double xl = 0.0;
                for (int l = 1; l <= 4; ++l) xl += SX(p, NREL(p, KX(i, j - 1), l));
                xl /= 4.0;
                SM(e, 1) = alfx * dzleft / fabs(xmean - xl);
            }
            if (j < nx) {
                double xr = 0.0;
                for (int l = 1; l <= 4; ++l) xr += SX(p, NREL(p, KX(i, j + 1), l));
                xr /= 4.0;
                double dum = alfx * dzright / fabs(xr - xmean);
                SM(e, 1) += dum;
                SM(e, 2) = -dum;
            }
            double dxup = fabs(SX(p, NREL(p, e, 3)) - SX(p, NREL(p, e, 4)));
            double dxdown = fabs(SX(p, NREL(p, e, 2)) - SX(p, NREL(p, e, 1)));
            double zmean = 0.0;
            for (int l = 1; l <= 4; ++l) zmean += SY(p, NREL(p, e, l));
            zmean /= 4.0;
            if (i > 1) {
                double zu = 0.0;
                for (int l = 1; l <= 4; ++l) zu += SY(p, NREL(p, KX(i - 1, j), l));
                zu /= 4.0;
                SM(e, 1) += alfz * dxup / fabs(zu - zmean);
            }
            if (i < nz) {
                double zd = 0.0;
                for (int l = 1; l <= 4; ++l) zd += SY(p, NREL(p, KX(i + 1, j), l));
                zd /= 4.0;
                double dum = alfz * dxdown / fabs(zmean - zd);
                SM(e, 1) += dum;
                SM(e, 3) = -dum;
            }
        }
#undef KX
#undef SM
}

/* ------------------------------------------------------------------------ */
/* Regulariser application R*(cgfac o p) (bp, src/cg_mod.f90:547-577, and
 * bptri, :579-613) or R*par (update.f90:63-106 with cg = NULL). */
static void orc_apply_R(const orc_cg_params *c, const dcplx *v, const double *cg, dcplx *out)
{
    const int manz = c->manz;
#define CGF(i) (cg ? cg[(i) - 1] : 1.0)
    if (c->ltri == 0) {
        const int nx = c->nx;
        const double *sm = c->smatm;
#define SM(m, k) sm[(size_t)((k) - 1) * manz + (m) - 1]
        for (int i = 1; i <= manz; ++i) {
            dcplx s = 0.0;
            if (i > 1) s = v[i - 2] * (SM(i - 1, 2) * CGF(i - 1));
            if (i < manz) s = s + v[i] * (SM(i, 2) * CGF(i + 1));
            if (i > nx) s = s + v[i - nx - 1] * (SM(i - nx, 3) * CGF(i - nx));
            if (i < manz - nx + 1) s = s + v[i + nx - 1] * (SM(i, 3) * CGF(i + nx));
            out[i - 1] = s + v[i - 1] * (SM(i, 1) * CGF(i));
        }
#undef SM
    } else {
        const int nnb = c->nnb;
        for (int i = 1; i <= manz; ++i) {
            dcplx s = 0.0;
            for (int j = 1; j <= nnb; ++j) {
                int id = c->nachbar[(size_t)(j - 1) * manz + i - 1];
                if (id != 0) {
                    if (cg)
                        s = s + v[id - 1] * c->smatm[(size_t)(j - 1) * manz + i - 1] * cg[id - 1];
                    else
                        s = s + c->smatm[(size_t)(j - 1) * manz + i - 1] * v[id - 1];
                }
            }
            if (cg)
                out[i - 1] = s + v[i - 1] * c->smatm[(size_t)nnb * manz + i - 1] * cg[i - 1];
            else
                out[i - 1] = s + c->smatm[(size_t)nnb * manz + i - 1] * v[i - 1];
        }
    }
#undef CGF
}

static double orc_Rdiag(const orc_cg_params *c, int j)
{
    if (c->ltri == 0) return c->smatm[j - 1];
    return c->smatm[(size_t)c->nnb * c->manz + j - 1];
}

/* src/cg_mod.f90:426-518 (cjggra) with bap :520-545, bp/bptri, bb :699-726 */
void orc_cjggra(const orc_cg_params *c, const dcplx *sens, const double *cgfac, dcplx *bvec,
                dcplx *dpar, double *cgres, int32_t *ncg_out)
{
    const int manz = c->manz, nanz = c->nanz;
    dcplx *rvec = (dcplx *)malloc(sizeof(dcplx) * manz);
    dcplx *pvec = (dcplx *)calloc(manz, sizeof(dcplx));
    dcplx *ap = (dcplx *)malloc(sizeof(dcplx) * nanz);
    double dr = 0, dr0 = 0, dr1 = 0, beta, alpha;
    int ncg = 0, k;
    for (int j = 0; j < manz; ++j) {
        dpar[j] = 0.0;
        rvec[j] = bvec[j];
    }
    for (k = 1; k <= c->ncgmax; ++k) {
        ncg = k - 1;
        dr = 0.0;
        for (int j = 0; j < manz; ++j) dr += creal(conj(rvec[j]) * rvec[j]);
        if (k == 1) {
            dr0 = dr * c->eps;
            beta = 0.0;
        } else {
            if (dr <= dr0) break;
            beta = dr / dr1;
        }
        for (int j = 0; j < manz; ++j) pvec[j] = rvec[j] + beta * pvec[j];
        /* bap: ap(i) = sum_j pvec(j)*sens(i,j)*cgfac(j)  (src/cg_mod.f90:520-545) */
        for (int i = 0; i < nanz; ++i) {
            dcplx s = 0.0;
            for (int j = 0; j < manz; ++j) s = s + pvec[j] * sens[(size_t)j * nanz + i] * cgfac[j];
            ap[i] = s;
        }
        orc_apply_R(c, pvec, cgfac, bvec);
        /* bb (src/cg_mod.f90:699-726) */
        for (int j = 0; j < manz; ++j) {
            dcplx s = 0.0;
            const dcplx *col = sens + (size_t)j * nanz;
            for (int i = 0; i < nanz; ++i) s = s + conj(col[i]) * (c->wmatd[i] * (double)c->wdfak[i]) * ap[i];
            bvec[j] = s + c->lam * bvec[j];
            bvec[j] = bvec[j] * cgfac[j];
        }
        dr1 = 0.0;
        for (int j = 0; j < manz; ++j) dr1 += creal(conj(pvec[j]) * bvec[j]);
        alpha = dr / dr1;
        for (int j = 0; j < manz; ++j) {
            dpar[j] = dpar[j] + alpha * pvec[j];
            rvec[j] = rvec[j] - alpha * bvec[j];
        }
        dr1 = dr;
        cgres[k] = (double)(float)(c->eps * dr / dr0);
    }
    if (k > c->ncgmax) ncg = c->ncgmax;
    cgres[0] = (double)(float)ncg;
    *ncg_out = ncg;
    free(rvec);
    free(pvec);
    free(ap);
}

/* src/cg_mod.f90:106-199 (cjggdc) with bapdc, bpdc/bpdctri, bbdc; the real
 * system uses sensdc (ldc) or the real part of sens (lfpi). */
void orc_cjggdc(const orc_cg_params *c, const dcplx *sens, const double *sensdc,
                const double *cgfac, dcplx *bvec, dcplx *dpar, double *cgres, int32_t *ncg_out)
{
    const int manz = c->manz, nanz = c->nanz;
    double *bv = (double *)malloc(sizeof(double) * manz);
    double *rv = (double *)malloc(sizeof(double) * manz);
    double *pv = (double *)calloc(manz, sizeof(double));
    double *ap = (double *)malloc(sizeof(double) * nanz);
    dcplx *tmp_in = (dcplx *)malloc(sizeof(dcplx) * manz);
    dcplx *tmp_out = (dcplx *)malloc(sizeof(dcplx) * manz);
#define JR(i, j) (c->ldc ? sensdc[(size_t)(j) * nanz + (i)] : creal(sens[(size_t)(j) * nanz + (i)]))
    for (int j = 0; j < manz; ++j) {
        bv[j] = c->lfpi ? cimag(bvec[j]) : creal(bvec[j]);
        dpar[j] = 0.0;
        rv[j] = bv[j];
    }
    double dr = 0, dr0 = 0, dr1 = 0, beta, alpha;
    int ncg = 0, k;
    for (k = 1; k <= c->ncgmax; ++k) {
        ncg = k - 1;
        dr = 0.0;
        for (int j = 0; j < manz; ++j) dr += rv[j] * rv[j];
        if (k == 1) {
            dr0 = dr * c->eps;
            beta = 0.0;
        } else {
            beta = dr / dr1;
        }
        if (dr <= dr0) break;
        for (int j = 0; j < manz; ++j) pv[j] = rv[j] + beta * pv[j];
        for (int i = 0; i < nanz; ++i) {
            double s = 0.0;
            for (int j = 0; j < manz; ++j) s = s + pv[j] * JR(i, j) * cgfac[j];
            ap[i] = s;
        }
        for (int j = 0; j < manz; ++j) tmp_in[j] = pv[j];
        orc_apply_R(c, tmp_in, cgfac, tmp_out);
        for (int j = 0; j < manz; ++j) {
            double s = 0.0;
            for (int i = 0; i < nanz; ++i) s = s + JR(i, j) * c->wmatd[i] * (double)c->wdfak[i] * ap[i];
            bv[j] = s + c->lam * creal(tmp_out[j]);
            bv[j] = bv[j] * cgfac[j];
        }
        dr1 = 0.0;
        for (int j = 0; j < manz; ++j) dr1 += pv[j] * bv[j];
        alpha = dr / dr1;
        for (int j = 0; j < manz; ++j) {
            dpar[j] = dpar[j] + alpha * pv[j];
            rv[j] = rv[j] - alpha * bv[j];
        }
        dr1 = dr;
        cgres[k] = (double)(float)(c->eps * dr / dr0);
    }
    if (k > c->ncgmax) ncg = c->ncgmax;
    cgres[0] = (double)(float)ncg;
    *ncg_out = ncg;
    for (int j = 0; j < manz; ++j) bvec[j] = bv[j];
#undef JR
    free(bv);
    free(rv);
    free(pv);
    free(ap);
    free(tmp_in);
    free(tmp_out);
}

/* src/update.f90:55-351 (lprior = ldiff = lw_ref = lphi0 = .false.) */
void orc_update(const orc_cg_params *c, const dcplx *sens, const double *sensdc, const dcplx *dat,
                const dcplx *sigmaa, double step, dcplx *par, dcplx *dpar, double *cgfac,
                dcplx *bvec_rhs, double *cgres, int32_t *ncg, double *bdpar)
{
    const int manz = c->manz, nanz = c->nanz;
    dcplx *bvec = (dcplx *)malloc(sizeof(dcplx) * manz);
    /* regularisation gradient R*par (update.f90:63-106) */
    orc_apply_R(c, par, NULL, bvec);
    for (int j = 0; j < manz; ++j) {
        double dum = 0.0;
        for (int i = 0; i < nanz; ++i) {
            double w = c->wmatd[i] * (double)c->wdfak[i];
            if (c->ldc) {
                double s = sensdc[(size_t)j * nanz + i];
                dum = dum + s * s * w;
            } else if (c->lfpi) {
                double s = creal(sens[(size_t)j * nanz + i]);
                dum = dum + s * s * w;
            } else {
                dcplx s = sens[(size_t)j * nanz + i];
                dum = dum + creal(conj(s) * s) * w;
            }
        }
        dum = dum + c->lam * orc_Rdiag(c, j + 1);
        cgfac[j] = 1.0 / sqrt(dum);
    }
    for (int j = 0; j < manz; ++j) {
        dcplx cd = 0.0;
        for (int i = 0; i < nanz; ++i) {
            double w = c->wmatd[i] * (double)c->wdfak[i];
            dcplx r = dat[i] - sigmaa[i];
            if (c->ldc)
                cd = cd + (sensdc[(size_t)j * nanz + i] * w) * r;
            else if (c->lfpi)
                cd = cd + (creal(sens[(size_t)j * nanz + i]) * w) * r;
            else
                cd = cd + conj(sens[(size_t)j * nanz + i]) * w * r;
        }
        bvec[j] = cd - c->lam * bvec[j];
        bvec[j] = bvec[j] * cgfac[j];
    }
    if (bvec_rhs) memcpy(bvec_rhs, bvec, sizeof(dcplx) * manz);
    if (c->ldc || c->lfpi)
        orc_cjggdc(c, sens, sensdc, cgfac, bvec, dpar, cgres, ncg);
    else
        orc_cjggra(c, sens, cgfac, bvec, dpar, cgres, ncg);
    if (c->lfpi)
        for (int j = 0; j < manz; ++j) dpar[j] = CMPLX(0.0, creal(dpar[j]));
    for (int j = 0; j < manz; ++j) dpar[j] = dpar[j] * cgfac[j];
    double bd = 0.0;
    for (int j = 0; j < manz; ++j) {
        par[j] = par[j] + step * dpar[j];
        bd = bd + creal(dpar[j] * conj(dpar[j]));
    }
    *bdpar = bd * step;
    free(bvec);
}

/* src/brough_mod.f90 (broughreg / broughtri, lprior = .false.) */
double orc_brough(const orc_cg_params *c, const dcplx *par)
{
    const int manz = c->manz;
    dcplx *rp = (dcplx *)malloc(sizeof(dcplx) * manz);
    orc_apply_R(c, par, NULL, rp);
    double rough = 0.0;
    for (int i = 0; i < manz; ++i) {
        if (c->lfpi)
            rough += cimag(rp[i]) * cimag(par[i]);
        else
            rough += creal(rp[i] * conj(par[i]));
    }
    free(rp);
    return rough;
}

/* src/dmisft.f90:73-137 with chkpo2 (:152-208) */
double orc_dmisft(int nanz, const dcplx *dat, const dcplx *sigmaa, const double *wmatd,
                  const double *wmatdr, const double *wmatdp, int lfpi, int lpol, double *betrms,
                  double *pharms, int32_t *npol)
{
    const double pi = acos(-1.0);
    double nrmsd = 0.0, br = 0.0, ph = 0.0;
    int idum = 0;
    for (int i = 0; i < nanz; ++i) {
        int wdlok = 1;
        double redat = creal(dat[i]), imdat = cimag(dat[i]);
        double resig = creal(sigmaa[i]), imsig = cimag(sigmaa[i]);
        int idat = imdat > pi / 2 ? -1 : (imdat <= -pi / 2 ? 1 : 0);
        int isig = imsig > pi / 2 ? -1 : (imsig <= -pi / 2 ? 1 : 0);
        if (idat == 0 && isig != 0) {
            imsig += (double)isig * pi;
            if (!lpol) imdat = imdat - copysign(pi, imdat);
            wdlok = 0;
        } else if (idat != 0 && isig == 0) {
            if (lpol) imdat = imdat + (double)idat * pi;
            wdlok = 0;
        } else if (idat != 0 && isig != 0) {
            imsig += (double)isig * pi;
            imdat += (double)idat * pi;
        }
        dcplx cd = CMPLX(redat, imdat) - CMPLX(resig, imsig);
        double psi = lfpi ? sqrt(wmatd[i]) * fabs(cimag(cd)) : sqrt(wmatd[i]) * cabs(cd);
        idum += wdlok;
        nrmsd += psi * psi * (double)wdlok;
        if (wmatdr) br += wmatdr[i] * (double)wdlok * creal(cd) * creal(cd);
        if (wmatdp) ph += wmatdp[i] * (double)wdlok * cimag(cd) * cimag(cd);
    }
    if (npol) *npol = nanz - idum;
    if (idum == 0) return -1.0;
    if (betrms) *betrms = sqrt(br / idum);
    if (pharms) *pharms = sqrt(ph / idum);
    return sqrt(nrmsd / (double)idum);
}

/* src/blam0.f90:131-167 (the Jacobian estimate, no preset): jtj(j) =
 * |sum_i sum_k conj(J_ij) J_ik w_i wdfak_i| (real parts for lfpi, sensdc
 * for ldc), lammax = 5 * 2/(alfx+alfz) * sum_j jtj(j) / manz.  The triple
 * loop of the reference, O(nanz manz^2): small problems only. */
double orc_blam0(const orc_cg_params *c, const dcplx *sens, const double *sensdc, double alfx, double alfz)
{
    const int M = c->manz, N = c->nanz;
    double tot = 0.0;
    for (int j = 0; j < M; ++j) {
        if (c->ldc || c->lfpi) {
            double dum = 0.0;
            for (int i = 0; i < N; ++i)
                for (int k = 0; k < M; ++k) {
                    const double a = c->ldc ? sensdc[i + (size_t)j * N] : creal(sens[i + (size_t)j * N]);
                    const double b = c->ldc ? sensdc[i + (size_t)k * N] : creal(sens[i + (size_t)k * N]);
                    dum += a * b * c->wmatd[i] * (double)c->wdfak[i];
                }
            tot += fabs(dum);
        } else {
            dcplx cdum = 0.0;
            for (int i = 0; i < N; ++i)
                for (int k = 0; k < M; ++k)
                    cdum += conj(sens[i + (size_t)j * N]) * sens[i + (size_t)k * N] *
                            (c->wmatd[i] * (double)c->wdfak[i]);
            tot += cabs(cdum);
        }
    }
    double lammax = tot / (double)M;
    lammax = lammax * 2.0 / (alfx + alfz);
    return lammax * 5.0;
}

/* src/parfit.f90:38-186: step length at the minimum of the parabola through
 * (0, fa), (0.5, fb), (1, fc), or where it crosses fmin, clamped to
 * [smin, 1]. */
double orc_parfit(double fa, double fb, double fc, double fmin, double smin)
{
    const double a = 0.0, b = 0.5, c = 1.0;
    double step = c;
#define ORC_PARAB() (b - ((b - a) * (b - a) * (fb - fc) - (b - c) * (b - c) * (fb - fa)) / \
                         (2.0 * ((b - a) * (fb - fc) - (b - c) * (fb - fa))))
    if (fa > fb) {
        if (fb <= fc) {
            if (fb <= fmin) {
                if (fa < fmin && fc > fa) step = b + (c - b) * (fmin - fb) / (fc - fb);
                else step = a + (b - a) * (fmin - fa) / (fb - fa);
            } else {
                step = ORC_PARAB();
            }
        } else {
            if (fb <= fmin) step = a + (b - a) * (fmin - fa) / (fb - fa);
            else if (fc <= fmin) step = b + (c - b) * (fmin - fb) / (fc - fb);
            else step = c;
        }
    } else if (fa < fb) {
        if (fb >= fc) {
            if (fb >= fmin) {
                if (fa > fmin && fc < fa) step = b + (c - b) * (fmin - fb) / (fc - fb);
                else step = a + (b - a) * (fmin - fa) / (fb - fa);
            } else {
                step = ORC_PARAB();
            }
        } else {
            if (fb >= fmin) step = a + (b - a) * (fmin - fa) / (fb - fa);
            else if (fc >= fmin) step = b + (c - b) * (fmin - fb) / (fc - fb);
            else step = c;
        }
    } else {
        if (fb > fc) {
            if (fb < fmin) step = ORC_PARAB();
            else if (fc <= fmin) step = b + (c - b) * (fmin - fb) / (fc - fb);
            else step = c;
        } else if (fb < fc) {
            if (fb > fmin) step = ORC_PARAB();
            else if (fc >= fmin) step = b + (c - b) * (fmin - fb) / (fc - fb);
            else step = c;
        } else {
            step = smin;
        }
    }
#undef ORC_PARAB
    if (step < smin) step = smin;
    return step > c ? c : step;
}
