// crt_cg.cu -- preconditioned CG on the Gauss-Newton normal equations.
//
// Restates cjggra (src/cg_mod.f90:426-518) and cjggdc (:106-199) with the
// operator pieces bap (J p, :520-545), bp / bptri (R p, :547-613) and bb
// (J^H W J p + lam R p, :699-726), and the set-up of src/update.f90:63-231
// (Jacobi factors cgfac and the scaled right-hand side).
//
// J is the sens(nanz, manz) array kept on the device as produced by the
// Jacobian kernel (column e contiguous in the readings i).  The two HBM
// passes per iteration are:
//   k_cg_jv  : ap_i = sum_e p_e J_ie cgfac_e     (threads over i, coalesced,
//              columns split into nsplit ranges, deterministic reduction)
//   k_cg_jhv : b_e  = (sum_i conj(J_ie) w_i ap_i + lam (R (cgfac o p))_e) cgfac_e
//              (one warp per 4 columns, w o ap staged per CTA)
// The FP64 dot products of an iteration's head and tail are formed by 32
// one-warp CTAs in the order of one 1024-thread CTA (the last to arrive adds
// the partials and takes the scalar step), the O(M) vector updates by
// grid-wide kernels; the lambda-batched solve keeps one CTA per candidate.
// The stop rule is evaluated on the device, so a batch of iterations can be
// queued without host round trips.  Real systems (DC, final phase
// improvement) use the same kernels with zero imaginary parts, which keeps
// the real arithmetic of cjggdc exact.
#include "crt_cg.h"

#include <cstdlib>
#include "crt_spc.h"
#include "crt_gnn.h"

namespace {

constexpr int VEC_NT = 1024;

// J(i, e) as an FP64 complex value: JP selects the storage precision,
// JM the Jacobian form (complex, real sensdc, real part of complex).
template <int JP, int JM>
__device__ __forceinline__ cd jval(const CGArgs& A, int e, int i)
{
    const size_t o = (size_t)e * A.N + i;
    if (JM == 1) {
        if (JP == 0) return cd{static_cast<const double*>(A.J)[o], 0.0};
        return cd{(double)static_cast<const float*>(A.J)[o], 0.0};
    }
    cd v;
    if (JP == 0) {
        v = static_cast<const cd*>(A.J)[o];
    } else {
        const cf f = static_cast<const cf*>(A.J)[o];
        v = cd{(double)f.x, (double)f.y};
    }
    if (JM == 2) v.y = 0.0;
    return v;
}

// J(i, e) in its storage type, converted by jcvt: lets a kernel keep a
// load in flight across a barrier and convert it afterwards.
template <int JP, int JM>
struct JRaw {
    using T = cd;
};
template <> struct JRaw<0, 1> { using T = double; };
template <> struct JRaw<1, 0> { using T = cf; };
template <> struct JRaw<1, 1> { using T = float; };
template <> struct JRaw<1, 2> { using T = cf; };

template <int JP, int JM>
__device__ __forceinline__ typename JRaw<JP, JM>::T jraw(const CGArgs& A, int e, int i)
{
    return static_cast<const typename JRaw<JP, JM>::T*>(A.J)[(size_t)e * A.N + i];
}

template <int JM>
__device__ __forceinline__ cd jcvt(cd v)
{
    if (JM == 2) v.y = 0.0;
    return v;
}
template <int JM>
__device__ __forceinline__ cd jcvt(cf f)
{
    return cd{(double)f.x, JM == 2 ? 0.0 : (double)f.y};
}
template <int JM>
__device__ __forceinline__ cd jcvt(double v) { return cd{v, 0.0}; }
template <int JM>
__device__ __forceinline__ cd jcvt(float v) { return cd{(double)v, 0.0}; }

// bp / bptri: (R (cgfac o p))_i
__device__ cd reg_apply_cg(const CGArgs& A, const cd* p, int i)
{
    const int M = A.M;
    const double* c = A.cgfac;
    if (A.ltri == 0) {
        const int nx = A.nx;
        const double *s1 = A.smatm, *s2 = s1 + M, *s3 = s2 + M;
        cd acc{0.0, 0.0};
        if (i > 0) acc = p[i - 1] * (s2[i - 1] * c[i - 1]);
        if (i < M - 1) acc = acc + p[i + 1] * (s2[i] * c[i + 1]);
        if (i >= nx) acc = acc + p[i - nx] * (s3[i - nx] * c[i - nx]);
        if (i < M - nx) acc = acc + p[i + nx] * (s3[i] * c[i + nx]);
        return acc + p[i] * (s1[i] * c[i]);
    }
    cd acc{0.0, 0.0};
    for (int j = 0; j < A.nnb; ++j) {
        const int id = A.nachbar[(size_t)j * M + i];
        if (id != 0) acc = acc + (p[id - 1] * A.smatm[(size_t)j * M + i]) * c[id - 1];
    }
    return acc + (p[i] * A.smatm[(size_t)A.nnb * M + i]) * c[i];
}

// update.f90:63-106: (R par)_i
__device__ cd reg_apply_par(const CGArgs& A, const cd* par, int i)
{
    const int M = A.M;
    if (A.ltri == 0) {
        const int nx = A.nx;
        const double *s1 = A.smatm, *s2 = s1 + M, *s3 = s2 + M;
        cd acc{0.0, 0.0};
        if (i > 0) acc = s2[i - 1] * par[i - 1];
        if (i < M - 1) acc = acc + s2[i] * par[i + 1];
        if (i >= nx) acc = acc + s3[i - nx] * par[i - nx];
        if (i < M - nx) acc = acc + s3[i] * par[i + nx];
        return acc + s1[i] * par[i];
    }
    cd acc{0.0, 0.0};
    for (int j = 0; j < A.nnb; ++j) {
        const int id = A.nachbar[(size_t)j * M + i];
        if (id != 0) acc = acc + A.smatm[(size_t)j * M + i] * par[id - 1];
    }
    return acc + A.smatm[(size_t)A.nnb * M + i] * par[i];
}

__device__ __forceinline__ double reg_diag(const CGArgs& A, int i)
{
    return A.ltri == 0 ? A.smatm[i] : A.smatm[(size_t)A.nnb * A.M + i];
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Butterfly reduction: every lane receives the warp's total.
__device__ __forceinline__ double warp_allsum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (all threads receive the total).
template <int NT>
__device__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < NT / 32 ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    double r = red[32];
    __syncthreads();
    return r;
}

// cgfac and scaled RHS: one warp per SU_COLS model cells, a CTA of SU_NT / 32
// warps; the readings' weights and residuals dat - sigmaa are staged in
// shared memory per chunk of SU_CHUNK readings (read once per CTA, not once
// per cell).  Lane l sums the rows l + 32 k in order, as one warp per cell
// would.
constexpr int SU_COLS = 4, SU_NT = 256, SU_CHUNK = 1024;

template <int JP, int JM>
__global__ void __launch_bounds__(SU_NT) k_cg_setup(CGArgs A, const cd* dat, const cd* sigmaa, const cd* par)
{
    using RT = typename JRaw<JP, JM>::T;
    __shared__ double s_w[SU_CHUNK];
    __shared__ cd s_rd[SU_CHUNK];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ebase = (blockIdx.x * (SU_NT / 32) + warp) * SU_COLS;
    const int nc = max(0, min(SU_COLS, A.M - ebase));
    const int N = A.N;
    double an[SU_COLS], arx[SU_COLS], ary[SU_COLS];
#pragma unroll
    for (int c = 0; c < SU_COLS; ++c) an[c] = arx[c] = ary[c] = 0.0;
    for (int r0 = 0; r0 < N; r0 += SU_CHUNK) {
        const int r1 = min(N, r0 + SU_CHUNK);
        __syncthreads();
        for (int t = threadIdx.x; t < r1 - r0; t += SU_NT) {
            s_w[t] = A.wd[r0 + t];
            s_rd[t] = dat[r0 + t] - sigmaa[r0 + t];
        }
        __syncthreads();
        if (nc == 0) continue;
        for (int i = r0 + lane; i < r1; i += 64) {
            RT j0[SU_COLS], j1[SU_COLS];
            const bool two = i + 32 < r1;
#pragma unroll
            for (int c = 0; c < SU_COLS; ++c) {
                j0[c] = c < nc ? jraw<JP, JM>(A, ebase + c, i) : RT{};
                j1[c] = (c < nc && two) ? jraw<JP, JM>(A, ebase + c, i + 32) : RT{};
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q == 1 && !two) break;
                const int ii = i + 32 * q - r0;
                const double w = s_w[ii];
                const cd rd = s_rd[ii];
#pragma unroll
                for (int c = 0; c < SU_COLS; ++c) {
                    const cd j = jcvt<JM>(q == 0 ? j0[c] : j1[c]);
                    an[c] += (j.x * j.x + j.y * j.y) * w;
                    const cd t = conj(j) * w * rd;
                    arx[c] += t.x;
                    ary[c] += t.y;
                }
            }
        }
    }
    if (nc == 0) return;
#pragma unroll
    for (int c = 0; c < SU_COLS; ++c) {
        an[c] = warp_sum(an[c]);
        arx[c] = warp_sum(arx[c]);
        ary[c] = warp_sum(ary[c]);
    }
    if (lane == 0) {
        for (int c = 0; c < nc; ++c) {
            const int e = ebase + c;
            const double dum = an[c] + A.lam * reg_diag(A, e);
            const double cg = 1.0 / sqrt(dum);
            A.cgfac[e] = cg;
            const cd rg = reg_apply_par(A, par, e);
            const cd b = cd{arx[c], ary[c]} - rg * A.lam;
            A.rhs[e] = b * cg;
        }
    }
}

__device__ void cg_init_body(const CGArgs& A)
{
    // cjggdc (src/cg_mod.f90:106-199) iterates on the real part of the
    // right-hand side (DC) or on its imaginary part (final phase improvement)
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        A.dpar[e] = cd{0.0, 0.0};
        const cd b = A.rhs[e];
        A.r[e] = A.jmode == 0 ? b : cd{A.jmode == 1 ? b.x : b.y, 0.0};
        A.p[e] = cd{0.0, 0.0};
        if (A.pc) A.rold[e] = cd{0.0, 0.0};
    }
    if (threadIdx.x == 0) {
        CGState s{};
        s.k = 1;
        s.done = A.ncgmax < 1;
        s.ncg = 0;
        *A.st = s;
    }
}

__global__ void __launch_bounds__(VEC_NT) k_cg_init(CGArgs A) { cg_init_body(A); }

// The head's scalar step (one thread): stop rule on dr = |r|^2 and
// beta = dr / dr1; returns 1 when the solve stops.
__device__ int head_decide(const CGArgs& A, double dr)
{
    CGState* st = A.st;
    const int k = st->k;
    int stop = 0;
    if (k == 1) {
        st->dr0 = dr * A.eps;
        // the real solver (cjggdc) tests the stop rule at k = 1 as well
        if (A.jmode != 0 && dr <= st->dr0) stop = 1;
    } else {
        if (dr <= st->dr0) stop = 1;
        st->beta = dr / st->dr1;
    }
    if (stop) {
        st->done = 1;
        st->ncg = k - 1;
    }
    st->dr = dr;
    st->num = dr;
    return stop;
}

// The preconditioned head's scalar step (one thread), see cg_begin_pc_body;
// returns 1 when the solve stops, *use_base whether the direction comes
// from the base preconditioner.
__device__ int head_pc_decide(const CGArgs& A, double dr, double gam_z, double gold_z, double gam_b, double gold_b,
                              int* use_base_out)
{
    CGState* st = A.st;
    const bool guard = A.pc_gnn != 0;
    const bool off0 = guard && st->no_gnn;
    const int k = st->k;
    int stop = 0;
    int use_base = off0 ? 1 : 0, restart = 0;
    if (guard && !off0) {
        bool bad = !(gam_z > 0.0);
        if (k == 1) st->dr_chk = dr;
        else if ((k - 1) % GNN_GUARD_WINDOW == 0) {
            if (dr > 0.5 * st->dr_chk) bad = true;
            st->dr_chk = dr;
        }
        if (bad) {
            st->no_gnn = 1;
            use_base = 1;
            restart = 1;
        }
    }
    const double gam = use_base ? gam_b : gam_z;
    const double gold = use_base ? gold_b : gold_z;
    double beta = 0.0;
    if (k == 1) {
        st->dr0 = dr * A.eps;
        if (A.jmode != 0 && dr <= st->dr0) stop = 1;
    } else {
        if (dr <= st->dr0) stop = 1;
        if (!restart) beta = (gam - gold) / st->gam;
    }
    if (stop) {
        st->done = 1;
        st->ncg = k - 1;
    }
    st->dr = dr;
    st->beta = beta;
    st->gam = gam;
    st->num = gam;
    *use_base_out = use_base;
    return stop;
}

// Iteration head: dr = |r|^2, stop rule, beta, p = r + beta p.
__device__ void cg_begin_body(const CGArgs& A)
{
    __shared__ double red[33];
    __shared__ int s_stop;
    CGState* st = A.st;
    if (st->done) return;
    double v = 0.0;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) v += cabs2(A.r[e]);
    const double dr = block_sum<VEC_NT>(v, red);
    const int k = st->k;
    double beta = 0.0;
    if (threadIdx.x == 0) s_stop = head_decide(A, dr);
    __syncthreads();
    if (s_stop) return;
    beta = (k == 1) ? 0.0 : st->beta;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) A.p[e] = A.r[e] + A.p[e] * beta;
}

// Preconditioned head: z (the preconditioner's output) is in A.z.  The stop
// rule is the reference's (|r|^2 against eps |r0|^2); beta is the flexible
// (Polak-Ribiere) Re(z^H (r - r_old)) / Re(z_old^H r_old), alpha's numerator
// Re(r^H z).  With the learned correction (pc_gnn) the head also guards it:
// a non-descent z or a stalled residual switches it off (no_gnn) and the
// direction restarts (beta = 0) from the base preconditioner's output.
__device__ void cg_begin_pc_body(const CGArgs& A)
{
    __shared__ double red[33];
    __shared__ int s_stop, s_base;
    __shared__ double s_beta;
    CGState* st = A.st;
    if (st->done) return;
    const bool guard = A.pc_gnn != 0;
    const bool off0 = guard && st->no_gnn;
    double v = 0.0, g = 0.0, go = 0.0, gb = 0.0, gob = 0.0;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        const cd r = A.r[e], ro = A.rold[e];
        v += cabs2(r);
        if (!off0) {
            const cd z = A.z[e];
            g += r.x * z.x + r.y * z.y;
            go += ro.x * z.x + ro.y * z.y;
        }
        if (guard) {
            const cd b = A.zb ? A.zb[e] : r;
            gb += r.x * b.x + r.y * b.y;
            gob += ro.x * b.x + ro.y * b.y;
        }
    }
    const double dr = block_sum<VEC_NT>(v, red);
    const double gam_z = block_sum<VEC_NT>(g, red);
    const double gold_z = block_sum<VEC_NT>(go, red);
    const double gam_b = guard ? block_sum<VEC_NT>(gb, red) : 0.0;
    const double gold_b = guard ? block_sum<VEC_NT>(gob, red) : 0.0;
    if (threadIdx.x == 0) {
        int use_base = 0;
        s_stop = head_pc_decide(A, dr, gam_z, gold_z, gam_b, gold_b, &use_base);
        s_beta = st->beta;
        s_base = use_base;
    }
    __syncthreads();
    if (s_stop) return;
    const double beta = s_beta;
    const bool base = s_base != 0;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        const cd r = A.r[e];
        const cd z = base ? (A.zb ? A.zb[e] : r) : A.z[e];
        A.p[e] = z + A.p[e] * beta;
        A.rold[e] = r;
    }
}

// ap partial sums over a column range: thread per reading.  The block stages
// p o cgfac for JV_CHUNK columns in shared memory and keeps JV_UNROLL
// independent J loads in flight per thread.
constexpr int JV_NT = 256, JV_CHUNK = 256, JV_UNROLL = 16;

template <int JP, int JM>
__global__ void __launch_bounds__(JV_NT) k_cg_jv(CGArgs A)
{
    __shared__ cd pcs[JV_CHUNK];
    if (A.st->done) return;
    const int i = blockIdx.x * JV_NT + threadIdx.x;
    const bool valid = i < A.N;
    const int split = blockIdx.y;
    const int per = (A.M + A.nsplit - 1) / A.nsplit;
    const int e0 = split * per, e1 = min(A.M, e0 + per);
    cd acc{0.0, 0.0};
    for (int eb = e0; eb < e1; eb += JV_CHUNK) {
        const int ne = min(JV_CHUNK, e1 - eb);
        __syncthreads();
        if ((int)threadIdx.x < ne) pcs[threadIdx.x] = A.p[eb + threadIdx.x] * A.cgfac[eb + threadIdx.x];
        __syncthreads();
        if (!valid) continue;
        int u = 0;
        for (; u + JV_UNROLL <= ne; u += JV_UNROLL) {
            cd jv[JV_UNROLL];
#pragma unroll
            for (int q = 0; q < JV_UNROLL; ++q) jv[q] = jval<JP, JM>(A, eb + u + q, i);
#pragma unroll
            for (int q = 0; q < JV_UNROLL; ++q) acc += pcs[u + q] * jv[q];
        }
        for (; u < ne; ++u) acc += pcs[u] * jval<JP, JM>(A, eb + u, i);
    }
    if (valid) A.part[(size_t)split * A.N + i] = acc;
}

// ap = sum of the partial sums; what the transposed product needs is w o ap.
__global__ void k_cg_jv_reduce(CGArgs A)
{
    if (A.st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.N) return;
    cd acc{0.0, 0.0};
    for (int s = 0; s < A.nsplit; ++s) acc += A.part[(size_t)s * A.N + i];
    A.ap[i] = acc * A.wd[i];
}

// b_e = (sum_i conj(J_ie) (w o ap)_i + lam (R (cgfac o p))_e) * cgfac_e,
// one warp per JH_COLS columns, a CTA of JH_NT / 32 warps.  Every warp reads
// all of w o ap, so the CTA stages it in shared memory in chunks of
// JH_CHUNK readings (cp.async, double-buffered): L2 serves w o ap once per
// CTA instead of once per warp.  Lane l sums the rows in pairs
// (l + 64 k, l + 64 k + 32), two pairs' loads in flight, then a rest of
// single rows past the last pair: the same order for every chunk size.
constexpr int JH_COLS = 4, JH_NT = 256, JH_CHUNK = 1024;

template <int JP, int JM, int NC = JH_COLS>
__global__ void __launch_bounds__(JH_NT) k_cg_jhv(CGArgs A)
{
    using RT = typename JRaw<JP, JM>::T;
    __shared__ __align__(16) cd s_ap[2][JH_CHUNK];
    if (A.st->done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ebase = (blockIdx.x * (JH_NT / 32) + warp) * NC;
    // warps past the last column still take part in the staging barriers
    const int nc = max(0, min(NC, A.M - ebase));
    const int N = A.N;
    auto stage = [&](int buf, int r0) {
        const int nr = min(JH_CHUNK, N - r0);
        for (int t = threadIdx.x; t < nr; t += JH_NT) cp_async16(&s_ap[buf][t], A.ap + r0 + t);
        cp_async_commit();
    };
    double ax[NC], ay[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        ax[c] = 0.0;
        ay[c] = 0.0;
    }
    auto pair = [&](const RT (&j0)[NC], const RT (&j1)[NC], cd w0, cd w1) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const cd t0 = conj(jcvt<JM>(j0[c])) * w0, t1 = conj(jcvt<JM>(j1[c])) * w1;
            ax[c] += t0.x + t1.x;
            ay[c] += t0.y + t1.y;
        }
    };
    auto ld = [&](RT (&dst)[NC], int i) {
#pragma unroll
        for (int c = 0; c < NC; ++c) dst[c] = c < nc ? jraw<JP, JM>(A, ebase + c, i) : RT{};
    };
    stage(0, 0);
    int buf = 0;
    for (int r0 = 0; r0 < N; r0 += JH_CHUNK, buf ^= 1) {
        if (r0 + JH_CHUNK < N) {
            stage(buf ^ 1, r0 + JH_CHUNK);
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();
        const int r1 = min(N, r0 + JH_CHUNK);
        const cd* w = s_ap[buf] - r0;
        int i = r0 + lane;
        if (nc > 0) {
            for (; i + 96 < r1; i += 128) {
                RT j0[NC], j1[NC], j2[NC], j3[NC];
                ld(j0, i);
                ld(j1, i + 32);
                ld(j2, i + 64);
                ld(j3, i + 96);
                pair(j0, j1, w[i], w[i + 32]);
                pair(j2, j3, w[i + 64], w[i + 96]);
            }
            for (; i + 32 < r1; i += 64) {
                RT j0[NC], j1[NC];
                ld(j0, i);
                ld(j1, i + 32);
                pair(j0, j1, w[i], w[i + 32]);
            }
            for (; i < r1; i += 32) {
                RT j0[NC];
                ld(j0, i);
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const cd t = conj(jcvt<JM>(j0[c])) * w[i];
                    ax[c] += t.x;
                    ay[c] += t.y;
                }
            }
        }
        __syncthreads();   // readers of `buf` are done before it is staged again
    }
    if (nc == 0) return;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        ax[c] = warp_allsum(ax[c]);
        ay[c] = warp_allsum(ay[c]);
    }
    if (lane < nc) {
        double bx = 0.0, by = 0.0;
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (c == lane) {
                bx = ax[c];
                by = ay[c];
            }
        const int e = ebase + lane;
        const cd rp = reg_apply_cg(A, A.p, e);
        const cd b = cd{bx, by} + rp * A.lam;
        A.bvec[e] = b * A.cgfac[e];
    }
}

// ---------------------------------------------------------------------------
// Fused matvec: b = (J^H (w o J p) + lam R (cgfac o p)) o cgfac from ONE read
// of J.  The kernel is persistent, one CTA per SM (cooperative launch, so
// every CTA is resident).  CTA c owns the column range [c per, (c+1) per);
// the readings are cut into row blocks of CGF_R.  Per block, the CTA copies
// its tile of J (per columns x CGF_R readings, complex64, 8-byte cp.async,
// CGF_S stages in flight) into shared memory and
//   1. forms its partial sums of (J p)_i over its columns and publishes
//      them to a ring slot; the CTA that arrives last at the slot adds the
//      grid's partials in CTA order (deterministic), multiplies by w and
//      releases the slot with the block's ticket;
//   2. one block later (the other CTAs' partials have arrived meanwhile)
//      waits for the previous block's ticket and accumulates
//      conj(J_ie) (w o J p)_i into its columns from the tile still held in
//      shared memory.
// A column's sum over the readings is formed in reading order, every
// reading's sum over the columns in a fixed order.  Waits are bounded:
// a wait that gives up sets *ferr and every CTA leaves.
// Tile layout: element (column e, reading r) of a stage at e * CGF_R +
// (r ^ (e & 15)), so the copies, the row-wise reads of step 1 and the
// column-wise reads of step 2 are all free of bank conflicts.
constexpr long CGF_POLL_LIMIT = 1L << 21;

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ cd ldcg_cd(const cd* p)
{
    const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}

__device__ __forceinline__ void stcg_cd(cd* p, cd v) { __stcg(reinterpret_cast<double2*>(p), make_double2(v.x, v.y)); }

// Thread 0: wait until the slot's ticket reaches `want`; false when the wait
// gave up (or another CTA's did).
__device__ bool cgf_wait(const CGArgs& A, const unsigned long long* flag, unsigned long long want)
{
    long polls = 0;
    while (ld_acquire_u64(flag) < want) {
        if (*(volatile int*)A.ferr) return false;
        if (++polls > CGF_POLL_LIMIT) {
            atomicExch(A.ferr, 1);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// Issue the copies of row block b into stage `st` (rows past N read as 0).
__device__ __forceinline__ void cgf_load(const CGArgs& A, cf* T, int e0, int ne, int b)
{
    const int i0 = b * CGF_R, nr = min(CGF_R, A.N - i0);
    const cf* J = static_cast<const cf*>(A.J);
    for (int idx = threadIdx.x; idx < ne * CGF_R; idx += CGF_NT) {
        const int e = idx >> 4, r = idx & 15;
        cf* dst = T + e * CGF_R + (r ^ (e & 15));
        if (r < nr) cp_async8(dst, J + (size_t)(e0 + e) * A.N + i0 + r);
        else *dst = cf{0.f, 0.f};
    }
}

template <int JM>
__global__ void __launch_bounds__(CGF_NT, 1) k_cg_fused(CGArgs A)
{
    extern __shared__ __align__(16) unsigned char cgf_smem[];
    __shared__ int s_last, s_ok;   // separate words: a slow warp may still read one after a barrier
    if (A.st->done) return;
    const int c = blockIdx.x, G = gridDim.x, tid = threadIdx.x;
    const int per = A.fper, e0 = c * per, ne = max(0, min(per, A.M - e0));
    const int nblk = (A.N + CGF_R - 1) / CGF_R;
    cf* tiles = reinterpret_cast<cf*>(cgf_smem);
    cd* pcs = reinterpret_cast<cd*>(tiles + (size_t)2 * CGF_S * per * CGF_R);
    cd* red = pcs + per;                  // [CGF_NT / CGF_R][CGF_R]
    cd* sv = red + CGF_NT;                // [CGF_R]
    const unsigned long long tbase = *A.fepoch * (unsigned long long)nblk;

    for (int t = tid; t < ne; t += CGF_NT) pcs[t] = A.p[e0 + t] * A.cgfac[e0 + t];
    // copy group g (one per iteration, CGF_S iterations ahead) holds the tile
    // of row block g for step 1 (stage g % CGF_S, from HBM) and that of
    // block g - L for step 2 (stage CGF_S + (g - L) % CGF_S, read again
    // while it is still in L2); L >= CGF_S, so the first groups hold no
    // step-2 tile
    const int L = A.flag_lag;
    auto vstage = [&](int blk) { return tiles + (size_t)(blk % CGF_S) * per * CGF_R; };
    auto hstage = [&](int blk) { return tiles + (size_t)(CGF_S + blk % CGF_S) * per * CGF_R; };
#pragma unroll
    for (int s = 0; s < CGF_S; ++s) {
        if (s < nblk) cgf_load(A, vstage(s), e0, ne, s);
        cp_async_commit();
    }
    cd acc{0.0, 0.0};
    const int g = tid >> 4, r = tid & 15;   // step 1: column group g, reading r
    bool ok = true;
    for (int b = 0; b < nblk + L; ++b) {
        cp_async_wait_group<CGF_S - 1>();
        __syncthreads();
        if (b < nblk) {
            // 1. partial sums of (J p)_i over this CTA's columns
            const cf* T = vstage(b);
            cd s{0.0, 0.0};
            for (int j = g; j < ne; j += CGF_NT / CGF_R) s += pcs[j] * jcvt<JM>(T[j * CGF_R + (r ^ (j & 15))]);
            red[g * CGF_R + r] = s;
            __syncthreads();
            const int slot = b % CGF_Q;
            if (tid < CGF_R) {
                cd t{0.0, 0.0};
                for (int q = 0; q < CGF_NT / CGF_R; ++q) t += red[q * CGF_R + tid];
                stcg_cd(A.fpart + ((size_t)slot * G + c) * CGF_R + tid, t);
                __threadfence();
            }
            __syncthreads();
            if (tid == 0) s_last = atomicAdd(A.fcnt + slot, 1) == G - 1;
            __syncthreads();
            if (s_last) {
                // the grid's partials of block b, added in CTA order
                __threadfence();
                cd t{0.0, 0.0};
                for (int q = g; q < G; q += CGF_NT / CGF_R) t += ldcg_cd(A.fpart + ((size_t)slot * G + q) * CGF_R + r);
                red[g * CGF_R + r] = t;
                __syncthreads();
                if (tid < CGF_R) {
                    cd ap{0.0, 0.0};
                    for (int q = 0; q < CGF_NT / CGF_R; ++q) ap += red[q * CGF_R + tid];
                    const int i = b * CGF_R + tid;
                    const cd v = i < A.N ? ap * A.wd[i] : cd{0.0, 0.0};
                    if (i < A.N) A.ap[i] = v;
                    stcg_cd(A.fv + (size_t)slot * CGF_R + tid, v);
                    __threadfence();
                }
                __syncthreads();
                if (tid == 0) {
                    A.fcnt[slot] = 0;
                    __threadfence();
                    st_release_u64(A.fflag + slot, tbase + (unsigned long long)b + 1ull);
                }
            }
        }
        const int h = b - L;
        if (h >= 0) {
            // 2. block h's w o (J p) (published while this CTA went on with
            // step 1 of later blocks), conj(J) times it into the columns
            const int slot = h % CGF_Q;
            if (tid == 0) {
                s_ok = cgf_wait(A, A.fflag + slot, tbase + (unsigned long long)h + 1ull);
                __threadfence();
            }
            __syncthreads();
            if (!s_ok) {
                ok = false;
                break;
            }
            if (tid < CGF_R) sv[tid] = ldcg_cd(A.fv + (size_t)slot * CGF_R + tid);
            __syncthreads();
            if (tid < ne) {
                const cf* T = hstage(h) + tid * CGF_R;
#pragma unroll
                for (int q = 0; q < CGF_R; ++q) acc += conj(jcvt<JM>(T[q ^ (tid & 15)])) * sv[q];
            }
        }
        __syncthreads();
        // the stages used in this iteration take the tiles of group b + CGF_S
        const int gn = b + CGF_S;
        if (gn < nblk) cgf_load(A, vstage(gn), e0, ne, gn);
        if (gn - L >= 0 && gn - L < nblk) cgf_load(A, hstage(gn - L), e0, ne, gn - L);
        cp_async_commit();
    }
    if (!ok) {
        cp_async_wait_all();
        return;
    }
    if (tid < ne) {
        const int e = e0 + tid;
        const cd rp = reg_apply_cg(A, A.p, e);
        A.bvec[e] = (acc + rp * A.lam) * A.cgfac[e];
    }
}

// The tail's scalar step (one thread) once alpha is known.
__device__ void tail_decide(const CGArgs& A, double alpha)
{
    CGState* st = A.st;
    const int k = st->k;
    st->alpha = alpha;
    st->dr1 = st->dr;
    A.cgres[k] = (double)(float)(A.eps * st->dr / st->dr0);
    st->k = k + 1;
    if (A.fused) *A.fepoch += 1;
    if (k + 1 > A.ncgmax) {
        st->done = 1;
        st->ncg = A.ncgmax;
    }
}

// Iteration tail: alpha = dr / Re(p^H b), dpar += alpha p, r -= alpha b.
__device__ void cg_end_body(const CGArgs& A)
{
    __shared__ double red[33];
    CGState* st = A.st;
    if (st->done) return;
    double v = 0.0;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        const cd pp = A.p[e], bb = A.bvec[e];
        v += pp.x * bb.x + pp.y * bb.y;
    }
    const double dr1 = block_sum<VEC_NT>(v, red);
    const double alpha = st->num / dr1;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        A.dpar[e] = A.dpar[e] + A.p[e] * alpha;
        A.r[e] = A.r[e] - A.bvec[e] * alpha;
    }
    if (threadIdx.x == 0) tail_decide(A, alpha);
}

// ---------------------------------------------------------------------------
// Head and tail of one solve across the grid.  CTA w (VEC_NT / 32 CTAs of one
// warp) forms the partial sums of warp w of the one-CTA form, element by
// element in the same order; the CTA that arrives last adds the partials as
// that form's final warp does and takes the scalar step, so every sum is
// formed in the one-CTA form's order (the lambda-batched solve still runs
// that form).  The vector updates then run as grid-wide kernels.
constexpr int VS_CTAS = VEC_NT / 32, VS_UPD_NT = 256;

// Lane 0 publishes q[0 .. n) of this CTA; true (in every lane) for the CTA
// that arrives last, which then finds the totals in tot[].
template <int n>
__device__ bool vs_gather(const CGArgs& A, const double (&q)[n], double (&tot)[n])
{
    const int lane = threadIdx.x;
    int last = 0;
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < n; ++j) __stcg(A.vred + blockIdx.x * 8 + j, q[j]);
        __threadfence();
        last = atomicAdd(&A.st->vcnt, 1) == VS_CTAS - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int j = 0; j < n; ++j) tot[j] = warp_sum(__ldcg(A.vred + lane * 8 + j));
    if (lane == 0) A.st->vcnt = 0;
    return true;
}

__global__ void __launch_bounds__(32) k_cg_head_sums(CGArgs A)
{
    if (A.st->done) return;
    double v = 0.0;
    for (int e = blockIdx.x * 32 + threadIdx.x; e < A.M; e += VEC_NT) v += cabs2(A.r[e]);
    const double q[1] = {warp_sum(v)};
    double tot[1];
    if (vs_gather<1>(A, q, tot) && threadIdx.x == 0) head_decide(A, tot[0]);
}

__global__ void __launch_bounds__(VS_UPD_NT) k_cg_head_update(CGArgs A)
{
    const CGState* st = A.st;
    if (st->done) return;
    const int e = blockIdx.x * VS_UPD_NT + threadIdx.x;
    if (e >= A.M) return;
    const double beta = (st->k == 1) ? 0.0 : st->beta;
    A.p[e] = A.r[e] + A.p[e] * beta;
}

__global__ void __launch_bounds__(32) k_cg_head_pc_sums(CGArgs A)
{
    CGState* st = A.st;
    if (st->done) return;
    const bool guard = A.pc_gnn != 0;
    const bool off0 = guard && st->no_gnn;
    double v = 0.0, g = 0.0, go = 0.0, gb = 0.0, gob = 0.0;
    for (int e = blockIdx.x * 32 + threadIdx.x; e < A.M; e += VEC_NT) {
        const cd r = A.r[e], ro = A.rold[e];
        v += cabs2(r);
        if (!off0) {
            const cd z = A.z[e];
            g += r.x * z.x + r.y * z.y;
            go += ro.x * z.x + ro.y * z.y;
        }
        if (guard) {
            const cd b = A.zb ? A.zb[e] : r;
            gb += r.x * b.x + r.y * b.y;
            gob += ro.x * b.x + ro.y * b.y;
        }
    }
    const double q[5] = {warp_sum(v), warp_sum(g), warp_sum(go), warp_sum(gb), warp_sum(gob)};
    double tot[5];
    if (vs_gather<5>(A, q, tot) && threadIdx.x == 0) {
        int use_base = 0;
        head_pc_decide(A, tot[0], tot[1], tot[2], guard ? tot[3] : 0.0, guard ? tot[4] : 0.0, &use_base);
        st->use_base = use_base;
    }
}

__global__ void __launch_bounds__(VS_UPD_NT) k_cg_head_pc_update(CGArgs A)
{
    const CGState* st = A.st;
    if (st->done) return;
    const int e = blockIdx.x * VS_UPD_NT + threadIdx.x;
    if (e >= A.M) return;
    const double beta = st->beta;
    const cd r = A.r[e];
    const cd z = st->use_base ? (A.zb ? A.zb[e] : r) : A.z[e];
    A.p[e] = z + A.p[e] * beta;
    A.rold[e] = r;
}

__global__ void __launch_bounds__(32) k_cg_tail_sums(CGArgs A)
{
    CGState* st = A.st;
    if (st->done) return;
    double v = 0.0;
    for (int e = blockIdx.x * 32 + threadIdx.x; e < A.M; e += VEC_NT) {
        const cd pp = A.p[e], bb = A.bvec[e];
        v += pp.x * bb.x + pp.y * bb.y;
    }
    const double q[1] = {warp_sum(v)};
    double tot[1];
    if (vs_gather<1>(A, q, tot) && threadIdx.x == 0) {
        tail_decide(A, st->num / tot[0]);
        st->pending = 1;
    }
}

// dpar += alpha p, r -= alpha b when the tail sums of this iteration ran
// (they may also have ended the solve at ncgmax); the last CTA to finish
// clears the flag.
__global__ void __launch_bounds__(VS_UPD_NT) k_cg_tail_update(CGArgs A)
{
    __shared__ int s_go;
    CGState* st = A.st;
    if (threadIdx.x == 0) s_go = st->pending;
    __syncthreads();
    if (!s_go) return;
    const double alpha = st->alpha;
    const int e = blockIdx.x * VS_UPD_NT + threadIdx.x;
    if (e < A.M) {
        A.dpar[e] = A.dpar[e] + A.p[e] * alpha;
        A.r[e] = A.r[e] - A.bvec[e] * alpha;
    }
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(&st->ucnt, 1) == (int)gridDim.x - 1) {
        st->ucnt = 0;
        st->pending = 0;
    }
}

__device__ void cg_finish_body(const CGArgs& A, int lfpi, double step, const cd* par_in, cd* par,
                               double* bdpar)
{
    __shared__ double red[33];
    double v = 0.0;
    for (int e = threadIdx.x; e < A.M; e += VEC_NT) {
        cd d = A.dpar[e];
        if (lfpi) d = cd{0.0, d.x};
        d = d * A.cgfac[e];
        A.dpar[e] = d;
        par[e] = par_in[e] + d * step;
        v += d.x * d.x + d.y * d.y;
    }
    const double s = block_sum<VEC_NT>(v, red);
    if (threadIdx.x == 0) {
        *bdpar = s * step;
        A.cgres[0] = (double)(float)A.st->ncg;
    }
}

__global__ void __launch_bounds__(VEC_NT) k_cg_finish(CGArgs A, int lfpi, double step, cd* par,
                                                      double* bdpar)
{
    cg_finish_body(A, lfpi, step, par, par, bdpar);
}

// ---------------------------------------------------------------------------
// Lambda candidates side by side (CGLArgs): the view of the buffers of the
// candidate in position k (slot L.slot[k]).
__device__ __forceinline__ CGArgs cgl_cand(const CGLArgs& L, int k)
{
    CGArgs A = L.a;
    const size_t M = (size_t)A.M, N = (size_t)A.N;
    const int b = L.slot[k];
    A.lam = L.lam[b];
    A.cgfac += b * M;
    A.rhs += b * M;
    A.p += b * M;
    A.r += b * M;
    A.bvec += b * M;
    A.dpar += b * M;
    A.z += b * M;
    A.rold += b * M;
    A.ap += b * N;
    A.part += (size_t)b * A.nsplit * N;
    A.cgres += (size_t)b * (A.ncgmax + 2);
    A.st += b;
    return A;
}

__device__ __forceinline__ bool cgl_all_done(const CGLArgs& L)
{
    for (int b = 0; b < L.nl; ++b)
        if (!L.a.st[L.slot[b]].done) return false;
    return true;
}

// k_cg_setup for every candidate: the sums over the readings do not depend
// on lambda and are formed once per cell.
template <int JP, int JM>
__global__ void k_cgl_setup(CGLArgs L, const cd* dat, const cd* sigmaa, const cd* par)
{
    const CGArgs& A = L.a;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= A.M) return;
    const int e = warp;
    double an = 0.0, arx = 0.0, ary = 0.0;
    for (int i = lane; i < A.N; i += 32) {
        const cd j = jval<JP, JM>(A, e, i);
        const double w = A.wd[i];
        const cd rd = dat[i] - sigmaa[i];
        an += (j.x * j.x + j.y * j.y) * w;
        const cd t = conj(j) * w * rd;
        arx += t.x;
        ary += t.y;
    }
    an = warp_sum(an);
    arx = warp_sum(arx);
    ary = warp_sum(ary);
    if (lane == 0) {
        const cd rg = reg_apply_par(A, par, e);
        for (int b = 0; b < L.nl; ++b) {
            const int sb = L.slot[b];
            const double lam = L.lam[sb];
            const double dum = an + lam * reg_diag(A, e);
            const double cg = 1.0 / sqrt(dum);
            A.cgfac[(size_t)sb * A.M + e] = cg;
            const cd rb = cd{arx, ary} - rg * lam;
            A.rhs[(size_t)sb * A.M + e] = rb * cg;
        }
    }
}

// One CTA per candidate for the O(M) vector work.
__global__ void __launch_bounds__(VEC_NT) k_cgl_init(CGLArgs L) { cg_init_body(cgl_cand(L, blockIdx.x)); }
__global__ void __launch_bounds__(VEC_NT) k_cgl_begin(CGLArgs L) { cg_begin_body(cgl_cand(L, blockIdx.x)); }
__global__ void __launch_bounds__(VEC_NT) k_cgl_begin_pc(CGLArgs L) { cg_begin_pc_body(cgl_cand(L, blockIdx.x)); }
__global__ void __launch_bounds__(VEC_NT) k_cgl_end(CGLArgs L) { cg_end_body(cgl_cand(L, blockIdx.x)); }
__global__ void __launch_bounds__(VEC_NT) k_cgl_finish(CGLArgs L, int lfpi, double step, const cd* par_in,
                                                       cd* par_out, double* bdpar)
{
    const int b = L.slot[blockIdx.x];
    cg_finish_body(cgl_cand(L, blockIdx.x), lfpi, step, par_in, par_out + (size_t)b * L.a.M, bdpar + b);
}

// k_cg_jv for NL candidates (slots b >= nl carry zeros): each J entry loaded
// once feeds NL accumulators.
template <int JP, int JM, int NL>
__global__ void __launch_bounds__(JV_NT) k_cgl_jv(CGLArgs L)
{
    __shared__ cd pcs[NL][JV_CHUNK];
    if (cgl_all_done(L)) return;
    const CGArgs& A = L.a;
    const size_t M = (size_t)A.M;
    const int i = blockIdx.x * JV_NT + threadIdx.x;
    const bool valid = i < A.N;
    const int split = blockIdx.y;
    const int per = (A.M + A.nsplit - 1) / A.nsplit;
    const int e0 = split * per, e1 = min(A.M, e0 + per);
    cd acc[NL];
#pragma unroll
    for (int b = 0; b < NL; ++b) acc[b] = cd{0.0, 0.0};
    for (int eb = e0; eb < e1; eb += JV_CHUNK) {
        const int ne = min(JV_CHUNK, e1 - eb);
        __syncthreads();
        if ((int)threadIdx.x < ne) {
            const int e = eb + threadIdx.x;
#pragma unroll
            for (int b = 0; b < NL; ++b)
                pcs[b][threadIdx.x] = b < L.nl ? A.p[L.slot[b] * M + e] * A.cgfac[L.slot[b] * M + e] : cd{0.0, 0.0};
        }
        __syncthreads();
        if (!valid) continue;
        int u = 0;
        for (; u + JV_UNROLL <= ne; u += JV_UNROLL) {
            cd jv[JV_UNROLL];
#pragma unroll
            for (int q = 0; q < JV_UNROLL; ++q) jv[q] = jval<JP, JM>(A, eb + u + q, i);
#pragma unroll
            for (int q = 0; q < JV_UNROLL; ++q) {
#pragma unroll
                for (int b = 0; b < NL; ++b) acc[b] += pcs[b][u + q] * jv[q];
            }
        }
        for (; u < ne; ++u) {
            const cd jv = jval<JP, JM>(A, eb + u, i);
#pragma unroll
            for (int b = 0; b < NL; ++b) acc[b] += pcs[b][u] * jv;
        }
    }
    if (!valid) return;
#pragma unroll
    for (int b = 0; b < NL; ++b)
        if (b < L.nl) A.part[((size_t)L.slot[b] * A.nsplit + split) * A.N + i] = acc[b];
}

// k_cg_jv_reduce per candidate (grid.y = candidate).
__global__ void k_cgl_jv_reduce(CGLArgs L)
{
    const CGArgs A = cgl_cand(L, blockIdx.y);
    if (A.st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.N) return;
    cd acc{0.0, 0.0};
    for (int s = 0; s < A.nsplit; ++s) acc += A.part[(size_t)s * A.N + i];
    A.ap[i] = acc * A.wd[i];
}

// k_cg_jhv for NL candidates: one warp per CglCols columns, a CTA of 8
// warps walks the readings in chunks of CglRows.  Every warp of the CTA
// needs the chunk's w o ap of all candidates, so the CTA stages it once in
// shared memory (cp.async, double-buffered); the J loads of the next chunk
// and its staging are issued before the current chunk is consumed, which
// keeps two chunks of loads in flight per warp.  Lane b * CglCols + c
// writes candidate b's column ebase + c.
constexpr int CGL_JH_NT = 256;
template <int NL>
struct CglCols {
    static constexpr int value = NL <= 2 ? 4 : (NL <= 4 ? 2 : 1);
};
template <int NL>
struct CglRows {   // two rows per lane with 4 columns, four otherwise (pairs of rows)
    static constexpr int value = NL <= 2 ? 64 : 128;
};

template <int JP, int JM, int NL>
__global__ void __launch_bounds__(CGL_JH_NT, 2) k_cgl_jhv(CGLArgs L)
{
    constexpr int NC = CglCols<NL>::value, RC = CglRows<NL>::value, RPL = RC / 32;
    static_assert(NL * NC <= 32, "one lane per (candidate, column)");
    using RT = typename JRaw<JP, JM>::T;
    __shared__ cd s_ap[2][NL][RC];
    if (cgl_all_done(L)) return;   // the same for every thread of the grid
    const CGArgs& A = L.a;
    const size_t N = (size_t)A.N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ebase = (blockIdx.x * (CGL_JH_NT / 32) + warp) * NC;
    // warps past the last column still take part in the staging barriers
    const int nc = max(0, min(NC, A.M - ebase));
    double ax[NL][NC], ay[NL][NC];
#pragma unroll
    for (int b = 0; b < NL; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            ax[b][c] = 0.0;
            ay[b][c] = 0.0;
        }
    // w o ap of rows r0 .. r0 + RC into buffer `buf`: copies for the entries
    // that exist, zeros for the rest (empty candidate slots, rows past N)
    auto stage = [&](int buf, int r0) {
        for (int t = threadIdx.x; t < NL * RC; t += CGL_JH_NT) {
            const int b = t / RC, rr = t - b * RC, i = r0 + rr;
            if (b < L.nl && i < A.N)
                cp_async16(&s_ap[buf][b][rr], A.ap + L.slot[b] * N + i);
            else
                s_ap[buf][b][rr] = cd{0.0, 0.0};
        }
        cp_async_commit();
    };
    auto load = [&](RT (&dst)[RPL][NC], int r0) {
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int i = r0 + q * 32 + lane;
#pragma unroll
            for (int c = 0; c < NC; ++c) dst[q][c] = (c < nc && i < A.N) ? jraw<JP, JM>(A, ebase + c, i) : RT{};
        }
    };
    RT jn[RPL][NC];
    load(jn, 0);
    stage(0, 0);
    int buf = 0;
    for (int r0 = 0; r0 < A.N; r0 += RC, buf ^= 1) {
        RT jr[RPL][NC];
#pragma unroll
        for (int q = 0; q < RPL; ++q)
#pragma unroll
            for (int c = 0; c < NC; ++c) jr[q][c] = jn[q][c];
        const bool more = r0 + RC < A.N;   // uniform over the CTA
        if (more) {
            // buffer buf ^ 1 was last read before the trailing barrier of
            // the previous chunk
            load(jn, r0 + RC);
            stage(buf ^ 1, r0 + RC);
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();   // chunk r0's w o ap is in shared memory
        // rows in pairs (lane + 64 k, lane + 64 k + 32) summed as k_cg_jhv
        // sums them; zero rows past N add exact zeros
#pragma unroll
        for (int q = 0; q < RPL; q += 2) {
#pragma unroll
            for (int b = 0; b < NL; ++b) {
                const cd w0 = s_ap[buf][b][q * 32 + lane], w1 = s_ap[buf][b][(q + 1) * 32 + lane];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const cd t0 = conj(jcvt<JM>(jr[q][c])) * w0, t1 = conj(jcvt<JM>(jr[q + 1][c])) * w1;
                    ax[b][c] += t0.x + t1.x;
                    ay[b][c] += t0.y + t1.y;
                }
            }
        }
        __syncthreads();   // readers of `buf` are done before it is staged again
    }
#pragma unroll
    for (int b = 0; b < NL; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            ax[b][c] = warp_allsum(ax[b][c]);
            ay[b][c] = warp_allsum(ay[b][c]);
        }
    const int mb = lane / NC, mc = lane % NC;
    if (mb < L.nl && mb < NL && mc < nc) {
        double bx = 0.0, by = 0.0;
#pragma unroll
        for (int b = 0; b < NL; ++b)
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (b == mb && c == mc) {
                    bx = ax[b][c];
                    by = ay[b][c];
                }
        const CGArgs C = cgl_cand(L, mb);
        const int e = ebase + mc;
        const cd rp = reg_apply_cg(C, C.p, e);
        const cd bv = cd{bx, by} + rp * C.lam;
        C.bvec[e] = bv * C.cgfac[e];
    }
}

}  // namespace

#define CRT_CG_DISPATCH(KERNEL, GRID, BLOCK, STREAM, ...)                          \
    do {                                                                           \
        const int key = a.jprec * 3 + a.jmode;                                     \
        switch (key) {                                                             \
        case 0: KERNEL<0, 0><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;      \
        case 1: KERNEL<0, 1><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;      \
        case 2: KERNEL<0, 2><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;      \
        case 3: KERNEL<1, 0><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;      \
        case 4: KERNEL<1, 1><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;      \
        default: KERNEL<1, 2><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;     \
        }                                                                          \
    } while (0)

void launch_cg_setup(const CGArgs& a, const cd* dat, const cd* sigmaa, const cd* par, cudaStream_t s)
{
    const int cols_per_block = (SU_NT / 32) * SU_COLS;
    CRT_CG_DISPATCH(k_cg_setup, (a.M + cols_per_block - 1) / cols_per_block, SU_NT, s, a, dat, sigmaa, par);
}

void launch_cg_init(const CGArgs& a, cudaStream_t s) { k_cg_init<<<1, VEC_NT, 0, s>>>(a); }

namespace {
// J^H pass with NC cells per warp (4; CRT_B200_JH_COLS=2 / 8 for the others)
template <int NC>
void launch_cg_jhv_nc(const CGArgs& a, cudaStream_t s)
{
    const int cols_per_block = (JH_NT / 32) * NC;
    const int grid = (a.M + cols_per_block - 1) / cols_per_block;
    switch (a.jprec * 3 + a.jmode) {
    case 0: k_cg_jhv<0, 0, NC><<<grid, JH_NT, 0, s>>>(a); break;
    case 1: k_cg_jhv<0, 1, NC><<<grid, JH_NT, 0, s>>>(a); break;
    case 2: k_cg_jhv<0, 2, NC><<<grid, JH_NT, 0, s>>>(a); break;
    case 3: k_cg_jhv<1, 0, NC><<<grid, JH_NT, 0, s>>>(a); break;
    case 4: k_cg_jhv<1, 1, NC><<<grid, JH_NT, 0, s>>>(a); break;
    default: k_cg_jhv<1, 2, NC><<<grid, JH_NT, 0, s>>>(a); break;
    }
}
void launch_cg_jhv(const CGArgs& a, cudaStream_t s)
{
    static const int nc = [] {
        const char* v = std::getenv("CRT_B200_JH_COLS");
        return v ? std::atoi(v) : JH_COLS;
    }();
    if (nc == 2) launch_cg_jhv_nc<2>(a, s);
    else if (nc == 8) launch_cg_jhv_nc<8>(a, s);
    else launch_cg_jhv_nc<4>(a, s);
}
}  // namespace

bool cg_fused_fits(const CGArgs& a, int grid, size_t smem_max)
{
    if (a.jprec != 1 || a.jmode == 1 || grid < 1) return false;
    const int per = (a.M + grid - 1) / grid;
    return per <= CGF_NT && cg_fused_smem(per) <= smem_max;
}

namespace {
void launch_cg_fused(const CGArgs& a, cudaStream_t s)
{
    const int grid = (a.M + a.fper - 1) / a.fper;
    const size_t smem = cg_fused_smem(a.fper);
    void* args[] = {const_cast<CGArgs*>(&a)};
    if (a.jmode == 2) {
        cudaFuncSetAttribute(k_cg_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaLaunchCooperativeKernel((const void*)k_cg_fused<2>, grid, CGF_NT, args, smem, s);
    } else {
        cudaFuncSetAttribute(k_cg_fused<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaLaunchCooperativeKernel((const void*)k_cg_fused<0>, grid, CGF_NT, args, smem, s);
    }
}
}  // namespace

void launch_cg_iterations(const CGArgs& a, int iters, const SpcPlan* spc, Gnn* gnn, cd* zb, cudaStream_t s)
{
    const int nt = 256;
    dim3 gjv((a.N + JV_NT - 1) / JV_NT, a.nsplit);
    const int gvec = (a.M + VS_UPD_NT - 1) / VS_UPD_NT;
    for (int it = 0; it < iters; ++it) {
        if (a.pc) {
            if (spc && gnn) {
                launch_spc_apply(*spc, a.r, zb, a.st, s);
                launch_gnn_apply(*gnn, a.r, zb, a.z, a.st, s);
            } else if (spc) {
                launch_spc_apply(*spc, a.r, a.z, a.st, s);
            } else {
                launch_gnn_apply(*gnn, a.r, nullptr, a.z, a.st, s);
            }
            k_cg_head_pc_sums<<<VS_CTAS, 32, 0, s>>>(a);
            k_cg_head_pc_update<<<gvec, VS_UPD_NT, 0, s>>>(a);
        } else {
            k_cg_head_sums<<<VS_CTAS, 32, 0, s>>>(a);
            k_cg_head_update<<<gvec, VS_UPD_NT, 0, s>>>(a);
        }
        if (a.fused) {
            launch_cg_fused(a, s);
        } else {
            CRT_CG_DISPATCH(k_cg_jv, gjv, JV_NT, s, a);
            k_cg_jv_reduce<<<(a.N + nt - 1) / nt, nt, 0, s>>>(a);
            launch_cg_jhv(a, s);
        }
        k_cg_tail_sums<<<VS_CTAS, 32, 0, s>>>(a);
        k_cg_tail_update<<<gvec, VS_UPD_NT, 0, s>>>(a);
    }
}

void launch_cg_finish(const CGArgs& a, int lfpi, double step, cd* par, double* bdpar, cudaStream_t s)
{
    k_cg_finish<<<1, VEC_NT, 0, s>>>(a, lfpi, step, par, bdpar);
}

// ---------------------------------------------------------------------------
// Lambda candidates side by side.
#define CRT_CGL_DISPATCH(KERNEL, NL, GRID, BLOCK, STREAM, ...)                     \
    do {                                                                           \
        const int key = L.a.jprec * 3 + L.a.jmode;                                 \
        switch (key) {                                                             \
        case 0: KERNEL<0, 0, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;  \
        case 1: KERNEL<0, 1, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;  \
        case 2: KERNEL<0, 2, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;  \
        case 3: KERNEL<1, 0, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;  \
        case 4: KERNEL<1, 1, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break;  \
        default: KERNEL<1, 2, NL><<<GRID, BLOCK, 0, STREAM>>>(__VA_ARGS__); break; \
        }                                                                          \
    } while (0)

namespace {

template <int NL>
void cgl_matvecs(const CGLArgs& L, cudaStream_t s)
{
    const CGArgs& a = L.a;
    const int nt = 256;
    const dim3 gjv((a.N + JV_NT - 1) / JV_NT, a.nsplit);
    CRT_CGL_DISPATCH(k_cgl_jv, NL, gjv, JV_NT, s, L);
    k_cgl_jv_reduce<<<dim3((a.N + nt - 1) / nt, L.nl), nt, 0, s>>>(L);
    const int cols_per_block = (CGL_JH_NT / 32) * CglCols<NL>::value;
    CRT_CGL_DISPATCH(k_cgl_jhv, NL, (a.M + cols_per_block - 1) / cols_per_block, CGL_JH_NT, s, L);
}

}  // namespace

void launch_cgl_setup(const CGLArgs& L, const cd* dat, const cd* sigmaa, const cd* par, cudaStream_t s)
{
    const CGArgs& a = L.a;
    const int threads = 256, warps = threads / 32;
    CRT_CG_DISPATCH(k_cgl_setup, (a.M + warps - 1) / warps, threads, s, L, dat, sigmaa, par);
}

void launch_cgl_init(const CGLArgs& L, cudaStream_t s) { k_cgl_init<<<L.nl, VEC_NT, 0, s>>>(L); }

int launch_cgl_iterations(const CGLArgs& L, int iters, cudaStream_t s)
{
    for (int it = 0; it < iters; ++it) {
        k_cgl_begin<<<L.nl, VEC_NT, 0, s>>>(L);
        if (L.nl <= 2)
            cgl_matvecs<2>(L, s);
        else if (L.nl <= 4)
            cgl_matvecs<4>(L, s);
        else
            cgl_matvecs<8>(L, s);
        k_cgl_end<<<L.nl, VEC_NT, 0, s>>>(L);
    }
    return 5 * iters;
}

int launch_cgl_iteration_pc(const CGLArgs& L, cudaStream_t s)
{
    k_cgl_begin_pc<<<L.nl, VEC_NT, 0, s>>>(L);
    if (L.nl <= 2)
        cgl_matvecs<2>(L, s);
    else if (L.nl <= 4)
        cgl_matvecs<4>(L, s);
    else
        cgl_matvecs<8>(L, s);
    k_cgl_end<<<L.nl, VEC_NT, 0, s>>>(L);
    return 5;
}

void launch_cgl_finish(const CGLArgs& L, int lfpi, double step, const cd* par_in, cd* par_out, double* bdpar,
                       cudaStream_t s)
{
    k_cgl_finish<<<L.nl, VEC_NT, 0, s>>>(L, lfpi, step, par_in, par_out, bdpar);
}
