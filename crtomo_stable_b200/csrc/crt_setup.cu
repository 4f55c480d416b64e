// crt_setup.cu -- set-up stage of the B200 path.
//
//  * crt_rwaven_host : wavenumbers and weights (src/rwaven.f90:49-151), FP64
//    on the host.
//  * k_elem_matrices / k_beta : the element stiffness-plus-mass matrices
//    elbg(e, imn, k) and the mixed-boundary coefficients kg(rel, l, k) of
//    src/precal.f90:57-208 (elem3/elem5/elem8/elem1/beta), one thread per
//    (element, wavenumber) or (boundary segment, electrode, wavenumber).
//  * build_assembly_lists : the gather form of kompab's scatter.  For every
//    band row i the non-zero entries (i, i-d) are listed with their
//    contributions in element order, so a row of the FE matrix can be formed
//    on the fly, in the reference's summation order, when it enters the
//    factorisation window.
#include "crt_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>

// ---------------------------------------------------------------------------
// Modified Bessel functions K0, K1 (with I0, I1): the Abramowitz & Stegun
// 9.8.1-9.8.8 polynomial approximations used by src/bessk0.f90 etc., with
// K0 = K1 = 0 beyond x = 500 as there.
__host__ __device__ static double bes_i0(double x)
{
    double ax = fabs(x);
    if (ax < 3.75) {
        double t = (x / 3.75) * (x / 3.75);
        return 1.0 + t * (3.5156229 + t * (3.0899424 + t * (1.2067492 + t * (0.2659732 +
               t * (0.360768e-1 + t * 0.45813e-2)))));
    }
    double t = 3.75 / ax;
    double poly = 0.39894228 + t * (0.1328592e-1 + t * (0.225319e-2 + t * (-0.157565e-2 +
                  t * (0.916281e-2 + t * (-0.2057706e-1 + t * (0.2635537e-1 + t * (-0.1647633e-1 +
                  t * 0.392377e-2)))))));
    return (exp(ax) / sqrt(ax)) * poly;
}

__host__ __device__ static double bes_i1(double x)
{
    double ax = fabs(x);
    if (ax < 3.75) {
        double t = (x / 3.75) * (x / 3.75);
        return x * (0.5 + t * (0.87890594 + t * (0.51498869 + t * (0.15084934 + t * (0.2658733e-1 +
               t * (0.301532e-2 + t * 0.32411e-3))))));
    }
    double t = 3.75 / ax;
    double poly = 0.39894228 + t * (-0.3988024e-1 + t * (-0.362018e-2 + t * (0.163801e-2 +
                  t * (-0.1031555e-1 + t * (0.2282967e-1 + t * (-0.2895312e-1 + t * (0.1787654e-1 +
                  t * -0.420059e-2)))))));
    return (exp(ax) / sqrt(ax)) * poly;
}

__host__ __device__ double crt_bessk0(double x)
{
    if (x <= 2.0) {
        double t = x * x / 4.0;
        return (-log(x / 2.0) * bes_i0(x)) + (-0.57721566 + t * (0.42278420 + t * (0.23069756 +
               t * (0.3488590e-1 + t * (0.262698e-2 + t * (0.10750e-3 + t * 0.74e-5))))));
    }
    if (x > 500.0) return 0.0;
    double t = 2.0 / x;
    return (exp(-x) / sqrt(x)) * (1.25331414 + t * (-0.7832358e-1 + t * (0.2189568e-1 +
           t * (-0.1062446e-1 + t * (0.587872e-2 + t * (-0.251540e-2 + t * 0.53208e-3))))));
}

__host__ __device__ double crt_bessk1(double x)
{
    if (x <= 2.0) {
        double t = x * x / 4.0;
        return (log(x / 2.0) * bes_i1(x)) + (1.0 / x) * (1.0 + t * (0.15443144 + t * (-0.67278579 +
               t * (-0.18156897 + t * (-0.1919402e-1 + t * (-0.110404e-2 + t * -0.4686e-4))))));
    }
    if (x > 500.0) return 0.0;
    double t = 2.0 / x;
    return (exp(-x) / sqrt(x)) * (1.25331414 + t * (0.23498619 + t * (-0.3655620e-1 +
           t * (0.1504268e-1 + t * (-0.780353e-2 + t * (0.325614e-2 + t * -0.68245e-3))))));
}

// ---------------------------------------------------------------------------
// Linear-triangle stiffness split into the three metric stencils and the
// consistent mass pattern (elem3; elem8 reuses them per sub-triangle).
__constant__ signed char c_tri_s1[9] = {1, -1, 0, -1, 1, 0, 0, 0, 0};
__constant__ signed char c_tri_s2[9] = {2, -1, -1, -1, 0, 1, -1, 1, 0};
__constant__ signed char c_tri_s3[9] = {1, 0, -1, 0, 0, 0, -1, 0, 1};
__constant__ signed char c_tri_s4[9] = {2, 1, 1, 1, 2, 1, 1, 1, 2};
// Bilinear quadrilateral (elem5) stencils.
__constant__ signed char c_q_s1[16] = {2, -2, -1, 1, -2, 2, 1, -1, -1, 1, 2, -2, 1, -1, -2, 2};
__constant__ signed char c_q_s2[16] = {1, 0, -1, 0, 0, -1, 0, 1, -1, 0, 1, 0, 0, 1, 0, -1};
__constant__ signed char c_q_s3[16] = {2, 1, -1, -2, 1, 2, -2, -1, -1, -2, 2, 1, -2, -1, 1, 2};
__constant__ signed char c_q_s4[16] = {4, 2, 1, 2, 2, 4, 2, 1, 1, 2, 4, 2, 2, 1, 2, 4};

// Metric coefficients of a triangle (p0, p1, p2); returns det.
__device__ static double tri_metric(double x0, double y0, double x1, double y1, double x2,
                                    double y2, double* a, double* b, double* c)
{
    double x21 = x1 - x0, x31 = x2 - x0, y21 = y1 - y0, y31 = y2 - y0;
    double det = x21 * y31 - x31 * y21;
    *a = (x31 * x31 + y31 * y31) / det;
    *b = -(x31 * x21 + y31 * y21) / det;
    *c = (x21 * x21 + y21 * y21) / det;
    return det;
}

// One thread per (area element, wavenumber): elbg[(k*E + e)*nmn + imn].
__global__ void k_elem_matrices(SetupArgs A)
{
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)A.E * A.K) return;
    const int e = (int)(t % A.E), k = (int)(t / A.E);
    const int typ = A.etyp[e], nk = A.enk[e];
    double xk[4], yk[4];
    for (int m = 0; m < nk; ++m) {
        int node = A.nrel0[e * A.maxnodes + m];
        int crd = A.snr0[node];
        xk[m] = A.sx[crd];
        yk[m] = A.sy[crd];
    }
    const double kw = A.kwn[k];
    double* out = A.elbg + ((int64_t)k * A.E + e) * A.nmn;
    if (typ == 3) {
        double a, b, c;
        double det = tri_metric(xk[0], yk[0], xk[1], yk[1], xk[2], yk[2], &a, &b, &c);
        if (det <= 0.0) { atomicMax(A.status, (int)CRT_ERR_ORIENT); return; }
        int imn = 0;
        for (int m = 0; m < 3; ++m)
            for (int q = 0; q <= m; ++q) {
                double mas = (a * c_tri_s1[m * 3 + q] + b * c_tri_s2[m * 3 + q] + c * c_tri_s3[m * 3 + q]) / 2.0;
                double mam = det * (double)c_tri_s4[m * 3 + q] / 2.4e1;
                out[imn++] = mas + mam * kw * kw;
            }
    } else if (typ == 5) {
        double x21 = xk[1] - xk[0], x31 = xk[3] - xk[0], y21 = yk[1] - yk[0], y31 = yk[3] - yk[0];
        double det = x21 * y31 - x31 * y21;
        if (det <= 0.0) { atomicMax(A.status, (int)CRT_ERR_ORIENT); return; }
        double a = (x31 * x31 + y31 * y31) / det, b = -(x31 * x21 + y31 * y21) / det,
               c = (x21 * x21 + y21 * y21) / det;
        int imn = 0;
        for (int m = 0; m < 4; ++m)
            for (int q = 0; q <= m; ++q) {
                double mas = (a * c_q_s1[m * 4 + q] + 3.0 * b * c_q_s2[m * 4 + q] + c * c_q_s3[m * 4 + q]) / 6.0;
                double mam = det * (double)c_q_s4[m * 4 + q] / 3.6e1;
                out[imn++] = mas + mam * kw * kw;
            }
    } else if (typ == 8) {
        // Four triangles around the intersection of the diagonals; the
        // centre node (index 4) is condensed out at this wavenumber.
        double a1 = xk[2] - xk[0], a2 = xk[3] - xk[1];
        if (fabs(a1) <= 1e-12 || fabs(a2) <= 1e-12) { atomicMax(A.status, (int)CRT_ERR_ORIENT); return; }
        a1 = (yk[2] - yk[0]) / a1;
        a2 = (yk[3] - yk[1]) / a2;
        if (fabs(a1 - a2) <= 1e-12) { atomicMax(A.status, (int)CRT_ERR_ORIENT); return; }
        double xd[5], yd[5];
        xd[4] = (a1 * xk[0] - yk[0] - a2 * xk[1] + yk[1]) / (a1 - a2);
        yd[4] = yk[0] + a1 * (xd[4] - xk[0]);
        for (int i = 0; i < 4; ++i) { xd[i] = xk[i]; yd[i] = yk[i]; }
        double S[25], M[25];
        for (int i = 0; i < 25; ++i) { S[i] = 0.0; M[i] = 0.0; }
        const int sub[4][3] = {{0, 1, 4}, {1, 2, 4}, {4, 2, 3}, {0, 4, 3}};
        for (int t4 = 0; t4 < 4; ++t4) {
            const int* ik = sub[t4];
            double a, b, c;
            double det = tri_metric(xd[ik[0]], yd[ik[0]], xd[ik[1]], yd[ik[1]], xd[ik[2]], yd[ik[2]], &a, &b, &c);
            if (det <= 1e-12) { atomicMax(A.status, (int)CRT_ERR_ORIENT); return; }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    S[ik[i] * 5 + ik[j]] += (a * c_tri_s1[i * 3 + j] + b * c_tri_s2[i * 3 + j] + c * c_tri_s3[i * 3 + j]) / 2.0;
                    M[ik[i] * 5 + ik[j]] += det * (double)c_tri_s4[i * 3 + j] / 2.4e1;
                }
        }
        for (int i = 0; i < 25; ++i) S[i] = S[i] + kw * kw * M[i];
        int imn = 0;
        for (int m = 0; m < 4; ++m)
            for (int q = 0; q <= m; ++q) out[imn++] = S[m * 5 + q] - S[m * 5 + 4] * S[4 * 5 + q] / S[24];
    } else {
        atomicMax(A.status, 18);
    }
}

// One thread per (mixed boundary segment, electrode, wavenumber):
// kg[(k*L + l)*R + rel] = beta(l, k) (src/beta.f90:69-121) and, from the
// first thread of every segment, relbg (elem1: L/6 [2 1; 1 2]).
__global__ void k_beta(SetupArgs A)
{
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t total = (int64_t)A.nmixed * A.L * A.K;
    if (t >= total) return;
    const int q = (int)(t % A.nmixed);
    const int l = (int)((t / A.nmixed) % A.L);
    const int k = (int)(t / ((int64_t)A.nmixed * A.L));
    const int rel = A.mixed_rel[q];              // 0-based boundary index
    const int ie = A.E + rel;                    // row in nrel
    int n0 = A.nrel0[ie * A.maxnodes + 0], n1 = A.nrel0[ie * A.maxnodes + 1];
    double x0 = A.sx[A.snr0[n0]], y0 = A.sy[A.snr0[n0]];
    double x1 = A.sx[A.snr0[n1]], y1 = A.sy[A.snr0[n1]];
    if (l == 0 && k == 0) {
        double x21 = x1 - x0, y21 = y1 - y0;
        double len = sqrt(x21 * x21 + y21 * y21);
        A.relbg[rel * 3 + 0] = len * 2.0 / 6.0;
        A.relbg[rel * 3 + 1] = len * 1.0 / 6.0;
        A.relbg[rel * 3 + 2] = len * 2.0 / 6.0;
    }
    const int en = A.snr0[A.enr0[l]];
    const double xs = A.sx[en], ys = A.sy[en];
    const double kw = A.kwn[k];
    double xr = (x0 + x1) / 2.0, yr = (y0 + y1) / 2.0;
    double x3 = xr - xs;
    double y3m = (yr - A.sytop) - (ys - A.sytop);
    double y3p = (yr - A.sytop) + (ys - A.sytop);
    double r1m = sqrt(x3 * x3 + y3m * y3m), r1p = sqrt(x3 * x3 + y3p * y3p);
    double x4 = y0 - y1, y4 = x1 - x0;
    double r2 = sqrt(x4 * x4 + y4 * y4);
    double out = 0.0;
    if (r1m < 1e-12 || r1p < 1e-12 || r2 < 1e-12) {
        atomicMax(A.status, (int)CRT_ERR_BETA);
    } else {
        double cm = (x3 * x4 + y3m * y4) / r1m / r2;
        double cp = (x3 * x4 + y3p * y4) / r1p / r2;
        double k0m = crt_bessk0(r1m * kw), k0p = crt_bessk0(r1p * kw);
        double k1m = crt_bessk1(r1m * kw), k1p = crt_bessk1(r1p * kw);
        double bt = (k0m + k0p == 0.0) ? (cm + cp) / 2.0 : (cm * k1m + cp * k1p) / (k0m + k0p);
        out = kw * bt;
    }
    A.kg[((int64_t)k * A.L + l) * A.R + rel] = out;
}

// ---------------------------------------------------------------------------
// Host side.

// Gauss-Legendre nodes/weights on [0, 1] and Gauss-Laguerre (alpha = 0),
// Newton iteration on the three-term recurrences (the methods of
// src/gauleg.f90 and src/gaulag.f90).
static void legendre_nodes(int n, double* x, double* w)
{
    const double x1 = 0.0, x2 = 1.0, xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        double z = std::cos(3.141592653589793 * ((double)i - 0.25) / ((double)n + 0.5)), z1, pp;
        for (;;) {
            double p0 = 1.0, pm = 0.0;
            for (int j = 1; j <= n; ++j) {
                double pmm = pm;
                pm = p0;
                p0 = ((2.0 * j - 1.0) * z * pm - ((double)j - 1.0) * pmm) / (double)j;
            }
            pp = (double)n * (z * p0 - pm) / (z * z - 1.0);
            z1 = z;
            z = z1 - p0 / pp;
            if (!(std::fabs(z - z1) > 3.0e-14)) break;
        }
        x[i - 1] = xm - xl * z;
        x[n - i] = xm + xl * z;
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
}

static void laguerre_nodes(int n, double* x, double* w)
{
    double z = 0.0;
    for (int i = 1; i <= n; ++i) {
        if (i == 1)
            z = 3.0 / (1.0 + 2.4 * n);
        else if (i == 2)
            z = z + 15.0 / (1.0 + 2.5 * n);
        else {
            double ai = (double)(i - 2);
            z = z + ((1.0 + 2.55 * ai) / (1.9 * ai)) * (z - x[i - 3]);
        }
        double p0 = 1.0, pm = 0.0, pp = 1.0;
        for (int it = 0; it < 10; ++it) {
            p0 = 1.0;
            pm = 0.0;
            for (int j = 1; j <= n; ++j) {
                double pmm = pm;
                pm = p0;
                p0 = (((double)(2 * j - 1) - z) * pm - (double)(j - 1) * pmm) / (double)j;
            }
            pp = ((double)n * p0 - (double)n * pm) / z;
            double z1 = z;
            z = z1 - p0 / pp;
            if (std::fabs(z - z1) <= 3.0e-14) break;
        }
        x[i - 1] = z;
        w[i - 1] = -1.0 / (pp * (double)n * pm);
    }
}

int crt_rwaven_host(int nanz, const int32_t* strnr, const int32_t* vnr, const int32_t* enr,
                    const int32_t* snr, const double* sx, const double* sy, int32_t* kwnanz,
                    double* kwn, double* kwnwi, double* amin_out, double* amax_out)
{
    double amin = 1e9, amax = 0.0;
    for (int i = 0; i < nanz; ++i) {
        int e[4] = {strnr[i] % 10000, strnr[i] / 10000, vnr[i] % 10000, vnr[i] / 10000};
        double xe[4] = {0, 0, 0, 0}, ye[4] = {0, 0, 0, 0};
        for (int j = 0; j < 4; ++j)
            if (e[j] > 0) {
                int c = snr[enr[e[j] - 1] - 1] - 1;
                xe[j] = sx[c];
                ye[j] = sy[c];
            }
        for (int v = 2; v < 4; ++v)
            for (int j = 0; j < 2; ++j)
                if (e[v] > 0 && e[j] > 0) {
                    double dx = xe[v] - xe[j], dy = ye[v] - ye[j];
                    double d = std::sqrt(dx * dx + dy * dy);
                    amin = std::min(d, amin);
                    amax = std::max(d, amax);
                }
    }
    if (amin_out) *amin_out = amin;
    if (amax_out) *amax_out = amax;
    if (amin < 1e-12 || amax < 1e-12) return CRT_ERR_TOPO;
    const int nlag = 4;
    int nleg = (int)(float)(6.0 * std::log10(amax / amin));   // int(real(...))
    nleg = std::min(std::max(nleg, 2), 30 - nlag);
    *kwnanz = nleg + nlag;
    const double k0 = 1.0 / (2.0 * amin);
    legendre_nodes(nleg, kwn, kwnwi);
    for (int i = 0; i < nleg; ++i) {
        kwnwi[i] = 2.0 * k0 * kwnwi[i] * kwn[i];
        kwn[i] = k0 * kwn[i] * kwn[i];
    }
    laguerre_nodes(nlag, kwn + nleg, kwnwi + nleg);
    for (int i = nleg; i < nleg + nlag; ++i) {
        kwnwi[i] = k0 * kwnwi[i] * std::exp(kwn[i]);
        kwn[i] = k0 * (kwn[i] + 1.0);
    }
    return CRT_OK;
}

// Running mean of the type-12 (no-flow) segment depths, src/bsytop.f90.
double crt_sytop_host(const MeshHost& m)
{
    double sytop = 0.0;
    int row = 0;
    for (int t = 0; t < m.typanz; ++t) {
        if (m.typ[t] == 12) {
            sytop = 0.0;
            for (int j = 1; j <= m.nelanz[t]; ++j, ++row) {
                double sp = 0.0;
                for (int q = 0; q < m.selanz[t]; ++q) {
                    int node = m.nrel[(size_t)q * m.ntot + row];
                    sp += m.sy[m.snr[node - 1] - 1];
                }
                sp /= (double)m.selanz[t];
                sytop = (j == 1) ? sp : (sytop * (double)(j - 1) + sp) / (double)j;
            }
        } else {
            row += m.nelanz[t];
        }
    }
    return sytop;
}

int build_assembly_lists(const MeshHost& m, AssemblyLists& out)
{
    struct Con { int row, d, code, sig; int64_t order; };
    std::vector<Con> cons;
    cons.reserve((size_t)m.elanz * 10 + (size_t)m.relanz * 3);
    int row = 0;
    int64_t order = 0;
    const int nmn = m.maxnodes * (m.maxnodes + 1) / 2;
    for (int t = 0; t < m.typanz; ++t) {
        const int ntyp = m.typ[t], nk = m.selanz[t];
        for (int j = 0; j < m.nelanz[t]; ++j, ++row) {
            if (ntyp > 11) continue;
            int ikl = 0;
            for (int a = 0; a < nk; ++a) {
                int nz = m.nrel[(size_t)a * m.ntot + row];
                for (int b = 0; b <= a; ++b) {
                    int nn = m.nrel[(size_t)b * m.ntot + row];
                    if (std::abs(nz - nn) > m.mb) return CRT_ERR_BAND;
                    Con c;
                    c.row = std::max(nz, nn) - 1;
                    c.d = std::abs(nz - nn);
                    if (ntyp == 11) {
                        int rel = row - m.elanz;             // 0-based
                        c.code = -(rel * 3 + ikl) - 1;
                        c.sig = m.rnr[rel] - 1;
                    } else {
                        c.code = row * nmn + ikl;
                        c.sig = row;
                    }
                    c.order = order++;
                    cons.push_back(c);
                    ++ikl;
                }
            }
        }
    }
    std::stable_sort(cons.begin(), cons.end(), [](const Con& x, const Con& y) {
        if (x.row != y.row) return x.row < y.row;
        if (x.d != y.d) return x.d < y.d;
        return x.order < y.order;
    });
    out.row_ptr.assign(m.sanz + 1, 0);
    out.ent_d.clear();
    out.ent_ptr.clear();
    out.con_code.clear();
    out.con_sig.clear();
    size_t i = 0;
    for (int r = 0; r < m.sanz; ++r) {
        out.row_ptr[r] = (int)out.ent_d.size();
        while (i < cons.size() && cons[i].row == r) {
            int d = cons[i].d;
            out.ent_d.push_back(d);
            out.ent_ptr.push_back((int)out.con_code.size());
            while (i < cons.size() && cons[i].row == r && cons[i].d == d) {
                out.con_code.push_back(cons[i].code);
                out.con_sig.push_back(cons[i].sig);
                ++i;
            }
        }
    }
    out.row_ptr[m.sanz] = (int)out.ent_d.size();
    out.ent_ptr.push_back((int)out.con_code.size());
    out.max_row_entries = 0;
    for (int r = 0; r < m.sanz; ++r)
        out.max_row_entries = std::max(out.max_row_entries, out.row_ptr[r + 1] - out.row_ptr[r]);
    return CRT_OK;
}
