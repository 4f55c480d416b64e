// crt_common.cuh -- shared device helpers for the CRTomo B200 path.
//
// Complex numbers are stored as two adjacent doubles (the layout of Fortran
// COMPLEX(KIND(0D0)) and C99 double _Complex).  Division follows Smith's
// algorithm (1962) and the square root is the principal branch, which are
// the rules gfortran applies to the reference's complex arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define CRT_HD __host__ __device__ __forceinline__

// entries of crt_last_timings_ex
#define CRT_NTIMINGS 18

struct __align__(16) cd {
    double x, y;
};

// complex64 storage element (the Jacobian in the mixed-precision form)
struct __align__(8) cf {
    float x, y;
};

CRT_HD cd mk(double x, double y) { return cd{x, y}; }
CRT_HD cf operator+(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }
CRT_HD cf operator-(cf a, cf b) { return cf{a.x - b.x, a.y - b.y}; }
CRT_HD cf operator-(cf a) { return cf{-a.x, -a.y}; }
CRT_HD cf operator*(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
CRT_HD cf& operator+=(cf& a, cf b) { a.x += b.x; a.y += b.y; return a; }
CRT_HD cf& operator-=(cf& a, cf b) { a.x -= b.x; a.y -= b.y; return a; }
CRT_HD cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
CRT_HD cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
CRT_HD cd operator-(cd a) { return cd{-a.x, -a.y}; }
CRT_HD cd operator*(cd a, cd b) { return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
CRT_HD cd operator*(cd a, double s) { return cd{a.x * s, a.y * s}; }
CRT_HD cd operator*(double s, cd a) { return cd{a.x * s, a.y * s}; }
CRT_HD cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }
CRT_HD cd& operator-=(cd& a, cd b) { a.x -= b.x; a.y -= b.y; return a; }
CRT_HD cd conj(cd a) { return cd{a.x, -a.y}; }
CRT_HD double cabs2(cd a) { return a.x * a.x + a.y * a.y; }

// Smith's complex division a / b.
CRT_HD cd cdiv(cd a, cd b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return cd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
    }
    double r = b.x / b.y, den = b.x * r + b.y;
    return cd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
}
CRT_HD cd operator/(cd a, cd b) { return cdiv(a, b); }
CRT_HD cd operator/(cd a, double s) { return cd{a.x / s, a.y / s}; }

// Principal square root: with r = |z|, t = sqrt((r + |Re z|)/2); the root
// is (t, Im z/(2t)) for Re z >= 0, else (|Im z|/(2t), copysign(t, Im z)).
CRT_HD cd csqrt_p(cd z)
{
    double r = hypot(z.x, z.y);
    if (r == 0.0) return cd{0.0, 0.0};
    double t = sqrt(0.5 * (r + fabs(z.x)));
    if (z.x >= 0.0) return cd{t, z.y / (2.0 * t)};
    return cd{fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}
CRT_HD double cabs_(cd a) { return hypot(a.x, a.y); }

// Scalar traits so kernels can be written once for the complex (kompab /
// chol / vre) and the real (kompadc / choldc / vredc) systems.
template <typename T> struct Sc;
template <> struct Sc<double> {
    static CRT_HD double zero() { return 0.0; }
    static CRT_HD double one() { return 1.0; }
    static CRT_HD double from(cd s) { return s.x; }            // DBLE(sigma)
    static CRT_HD double absval(double a) { return a; }       // scaldc tests a <= 0
    static CRT_HD double normalise(double a, double) { return 1.0; }
    static CRT_HD double sqrt_(double a) { return sqrt(a); }
    static CRT_HD double sqrt_fast(double a) { return sqrt(a); }
    static CRT_HD bool bad_pivot(double s) { return !(s > 0.0); }
    // root = sqrt(z) and inv = 1 / root from one reciprocal square root
    static __device__ __forceinline__ void sqrt_recip(double z, double& root, double& inv)
    {
        inv = rsqrt(z);
        root = z * inv;
    }
    static CRT_HD double mul(double a, double b) { return a * b; }
    static CRT_HD double div(double a, double b) { return a / b; }
    static CRT_HD double recip(double a) { return 1.0 / a; }
    static CRT_HD cd to_cd(double a) { return cd{a, 0.0}; }
};
template <> struct Sc<cd> {
    static CRT_HD cd zero() { return cd{0.0, 0.0}; }
    static CRT_HD cd one() { return cd{1.0, 0.0}; }
    static CRT_HD cd from(cd s) { return s; }
    static CRT_HD double absval(cd a) { return cabs_(a); }
    static CRT_HD cd normalise(cd a, double d) { return cd{a.x / d, a.y / d}; }
    static CRT_HD cd sqrt_(cd a) { return csqrt_p(a); }
    // principal root with |z| = sqrt(x^2 + y^2) (no overflow scaling; the
    // pivots of the scaled systems are of order one)
    static CRT_HD cd sqrt_fast(cd z)
    {
        const double r = sqrt(z.x * z.x + z.y * z.y);
        if (r == 0.0) return cd{0.0, 0.0};
        const double t = sqrt(0.5 * (r + fabs(z.x)));
        const double h = 0.5 / t;
        if (z.x >= 0.0) return cd{t, z.y * h};
        return cd{fabs(z.y) * h, copysign(t, z.y)};
    }
    static CRT_HD bool bad_pivot(cd s) { return !(s.x * s.x + s.y * s.y > 0.0); }
    // Principal root of z and its reciprocal from two reciprocal square
    // roots and no division: with r = |z|, t = sqrt((r + |Re z|)/2) the root
    // is (t, Im z/(2t)) or (|Im z|/(2t), copysign(t, Im z)), and since
    // |root|^2 = r, 1/root = conj(root)/r.
    static __device__ __forceinline__ void sqrt_recip(cd z, cd& root, cd& inv)
    {
        const double r2 = z.x * z.x + z.y * z.y;
        if (!(r2 > 0.0)) {
            root = cd{0.0, 0.0};
            inv = cd{0.0, 0.0};
            return;
        }
        const double ir = rsqrt(r2), r = r2 * ir;
        const double u = 0.5 * (r + fabs(z.x));
        const double iu = rsqrt(u), t = u * iu, h = 0.5 * iu;
        root = z.x >= 0.0 ? cd{t, z.y * h} : cd{fabs(z.y) * h, copysign(t, z.y)};
        inv = cd{root.x * ir, -root.y * ir};
    }
    static CRT_HD cd mul(cd a, cd b) { return a * b; }
    static CRT_HD cd div(cd a, cd b) { return cdiv(a, b); }
    // 1/a = conj(a) / |a|^2 (the pivots are of order one after scaling)
    static CRT_HD cd recip(cd a)
    {
        const double s = 1.0 / (a.x * a.x + a.y * a.y);
        return cd{a.x * s, -a.y * s};
    }
    static CRT_HD cd to_cd(cd a) { return a; }
};

// acc -= a * b as fused multiply-adds (4 for complex operands, 1 for real)
CRT_HD void fms_acc(cd& acc, cd a, cd b)
{
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}
CRT_HD void fms_acc(double& acc, double a, double b) { acc = fma(-a, b, acc); }

CRT_HD void fms_acc(cf& acc, cf a, cf b)
{
    acc.x = fmaf(-a.x, b.x, acc.x);
    acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(-a.x, b.y, acc.y);
    acc.y = fmaf(-a.y, b.x, acc.y);
}
CRT_HD cf scale(cf a, double s) { return cf{(float)(a.x * s), (float)(a.y * s)}; }

CRT_HD double scale(double a, double s) { return a * s; }
CRT_HD cd scale(cd a, double s) { return cd{a.x * s, a.y * s}; }

// complex64 storage and arithmetic of the mixed-precision factorisation
// (the quantities it is formed from are computed in FP64, see crt_band_blk.cu)
template <> struct Sc<cf> {
    static CRT_HD cf zero() { return cf{0.0f, 0.0f}; }
    static CRT_HD cf one() { return cf{1.0f, 0.0f}; }
    static CRT_HD cf from(cd s) { return cf{(float)s.x, (float)s.y}; }
    static CRT_HD double absval(cf a) { return hypot((double)a.x, (double)a.y); }
    static CRT_HD cf normalise(cf a, double d) { return cf{(float)(a.x / d), (float)(a.y / d)}; }
    static CRT_HD bool bad_pivot(cf s) { return !(s.x * s.x + s.y * s.y > 0.0f); }
    static __device__ __forceinline__ void sqrt_recip(cf z, cf& root, cf& inv)
    {
        const float r2 = z.x * z.x + z.y * z.y;
        if (!(r2 > 0.0f)) {
            root = cf{0.0f, 0.0f};
            inv = cf{0.0f, 0.0f};
            return;
        }
        const float ir = rsqrtf(r2), r = r2 * ir;
        const float u = 0.5f * (r + fabsf(z.x));
        const float iu = rsqrtf(u), t = u * iu, h = 0.5f * iu;
        root = z.x >= 0.0f ? cf{t, z.y * h} : cf{fabsf(z.y) * h, copysignf(t, z.y)};
        inv = cf{root.x * ir, -root.y * ir};
    }
    static CRT_HD cf mul(cf a, cf b) { return a * b; }
    static CRT_HD cf recip(cf a)
    {
        const float s = 1.0f / (a.x * a.x + a.y * a.y);
        return cf{a.x * s, -a.y * s};
    }
    static CRT_HD cd to_cd(cf a) { return cd{(double)a.x, (double)a.y}; }
};

// FP64 type in which a storage type's values are formed
template <typename T> struct Wide { using type = T; };
template <> struct Wide<cf> { using type = cd; };
template <typename T> CRT_HD T narrow(typename Wide<T>::type v);
template <> CRT_HD double narrow<double>(double v) { return v; }
template <> CRT_HD cd narrow<cd>(cd v) { return v; }
template <> CRT_HD cf narrow<cf>(cd v) { return cf{(float)v.x, (float)v.y}; }

// 16-byte asynchronous global -> shared copies (cp.async, bypassing L1);
// both addresses 16-byte aligned.  wait_group<N> returns once at most N of
// the thread's committed groups are still in flight.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { cp_async_wait_group<0>(); }

// mbarrier and bulk-copy (TMA engine, untiled) helpers: one CTA, no cluster
// multicast.  The wait gives up after a bounded number of polls and
// reports failure instead of spinning for ever.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, int bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, int bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, int phase)
{
    const unsigned a = smem_u32(bar);
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Reference error numbers (src/error.txt) returned through the C ABI.
enum crt_errnr : int32_t {
    CRT_OK = 0,
    CRT_ERR_BAND = 19,        // kompab: |i-j| > mb
    CRT_ERR_ORIENT = 26,      // elem3/elem8: bad element orientation
    CRT_ERR_ZERO_DIAG = 27,   // scalab/scaldc: zero diagonal
    CRT_ERR_PIVOT = 28,       // chol/choldc: non-positive pivot
    CRT_ERR_BETA = 35,        // beta: degenerate boundary geometry
    CRT_ERR_TOPO = 73,        // rwaven: duplicate electrodes
    CRT_ERR_ZERO_VOLT = 82,   // bvolti: zero voltage
    CRT_ERR_KFAK = 93,        // bkfak: zero geometric factor
    CRT_ERR_ALLOC = 97,       // allocation problem
    CRT_ERR_ARG = 3,          // inconsistent input
    CRT_ERR_CUDA = 200,       // CUDA runtime failure (no reference counterpart)
    CRT_ERR_UNSUPPORTED = 201 // option outside the implemented path
};
