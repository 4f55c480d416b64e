// crt_schur.cu -- forward model by elimination of the mixed-boundary nodes
// (see crt_schur.h for the algebra).  Kernels, in the order they run:
//
//   k_schur_rhs_src / k_schur_rhs_cpl  the columns F r_I (one per source
//       electrode) and F A_IG (one per boundary node) of the interior
//       solves, and the coupling values a(g, i) kept for later steps;
//   k_schur_transpose  the interior factor reversed and row-packed, so the
//       back substitution runs as a forward sweep;
//   k_schur_sweep   banded triangular sweep of R columns per CTA (forward for
//       all columns, each block from its first non-zero row; back for the
//       source columns): the factor streams through shared memory in blocks
//       of 16 columns (one bulk copy each, double-buffered, bounded
//       mbarrier wait), the right-hand sides in a window of rows that arrive
//       by cp.async two blocks ahead; per block a 16-row triangle (half-warp
//       per column, shuffle broadcasts) and an (mb x 16) x (16 x R) update
//       in 4 x 4 register tiles;
//   k_schur_gram    C = V^T [u^ | V^] per wavenumber (tiled GEMM that skips
//       the rows where a column is still zero);
//   k_schur_chol    per (k, l): S_l = A_GG(l) - V^T V^, right-looking
//       blocked Cholesky (unconjugated, complex symmetric as
//       src/chol.f90:44-78) with a 16-column panel in shared memory, the
//       forward solve fused into the factorisation, the back solve by panels;
//   k_schur_zrebuild  z^ = u^ - V^ p_G (tiled GEMM);
//   k_schur_out_gam p_G into kpot at the boundary nodes.
#include "crt_schur.h"

#include <cstdlib>
#include <cstring>

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <utility>

// ---------------------------------------------------------------------------
// Host plan.
int schur_plan_host(const AssemblyLists& full, int n, const std::vector<int>& gamma_nodes,
                    const std::vector<int>& enr0, int lsink, int nsink0, SchurHost& o, int R)
{
    o = SchurHost{};
    o.R = R;
    o.n = n;
    o.L = (int)enr0.size();
    std::vector<int> posI(n, -1), posG(n, -1);
    std::vector<char> isg(n, 0);
    for (int v : gamma_nodes)
        if (v >= 0 && v < n) isg[v] = 1;
    for (int v = 0; v < n; ++v) {
        if (isg[v]) {
            posG[v] = (int)o.gam.size();
            o.gam.push_back(v);
        } else {
            posI[v] = (int)o.permI.size();
            o.permI.push_back(v);
        }
    }
    o.nI = (int)o.permI.size();
    o.m = (int)o.gam.size();
    if (o.nI == 0 || o.m == 0 || o.m > SCHUR_MMAX) return CRT_ERR_ARG;
    AssemblyLists& li = o.lists_I;
    li.row_ptr.assign(1, 0);
    li.ent_ptr.assign(1, 0);
    std::vector<std::vector<std::pair<int, int>>> cpl(o.m);   // per g: (interior position, gather entry)
    for (int r = 0; r < n; ++r) {
        const int pr = posI[r];
        for (int e = full.row_ptr[r]; e < full.row_ptr[r + 1]; ++e) {
            const int c = r - full.ent_d[e];
            if (pr >= 0 && posI[c] >= 0) {
                li.ent_d.push_back(pr - posI[c]);
                for (int q = full.ent_ptr[e]; q < full.ent_ptr[e + 1]; ++q) {
                    // a mixed-boundary segment couples boundary nodes only
                    if (full.con_code[q] < 0) return CRT_ERR_ARG;
                    li.con_code.push_back(full.con_code[q]);
                    li.con_sig.push_back(full.con_sig[q]);
                }
                li.ent_ptr.push_back((int)li.con_code.size());
                o.mbI = std::max(o.mbI, pr - posI[c]);
            } else if (pr >= 0) {
                cpl[posG[c]].push_back({pr, e});
            } else if (posI[c] >= 0) {
                cpl[posG[r]].push_back({posI[c], e});
            } else {
                o.gg_g.push_back(posG[r]);   // r >= c, so g >= h
                o.gg_h.push_back(posG[c]);
                o.gg_ent.push_back(e);
            }
        }
        if (pr >= 0) {
            li.row_ptr.push_back((int)li.ent_d.size());
            li.max_row_entries = std::max(li.max_row_entries, li.row_ptr.back() - li.row_ptr[li.row_ptr.size() - 2]);
        }
    }
    // rows of D_l: the G-G entries with a mixed-boundary contribution, both
    // triangles, by row
    {
        std::vector<std::vector<std::pair<int, int>>> bd(o.m);
        for (size_t q = 0; q < o.gg_ent.size(); ++q) {
            const int e = o.gg_ent[q];
            bool mixed = false;
            for (int c = full.ent_ptr[e]; c < full.ent_ptr[e + 1]; ++c) mixed |= full.con_code[c] < 0;
            if (!mixed) continue;
            bd[o.gg_g[q]].push_back({o.gg_h[q], e});
            if (o.gg_g[q] != o.gg_h[q]) bd[o.gg_h[q]].push_back({o.gg_g[q], e});
        }
        o.bd_ptr.assign(1, 0);
        for (int g = 0; g < o.m; ++g) {
            std::sort(bd[g].begin(), bd[g].end());
            for (auto& he : bd[g]) {
                o.bd_col.push_back(he.first);
                o.bd_ent.push_back(he.second);
            }
            o.bd_ptr.push_back((int)o.bd_col.size());
        }
    }
    o.gi_ptr.assign(1, 0);
    std::vector<int> first(o.L + o.m, o.nI);
    for (int g = 0; g < o.m; ++g) {
        std::sort(cpl[g].begin(), cpl[g].end());
        for (auto& pe : cpl[g]) {
            o.gi_pos.push_back(pe.first);
            o.gi_ent.push_back(pe.second);
            o.gi_g.push_back(g);
            first[o.L + g] = std::min(first[o.L + g], pe.first);
        }
        o.gi_ptr.push_back((int)o.gi_pos.size());
    }
    o.posI_src.resize(o.L);
    o.posG_src.resize(o.L);
    o.posI_sink = lsink ? posI[nsink0] : -1;
    o.posG_sink = lsink ? posG[nsink0] : -1;
    for (int l = 0; l < o.L; ++l) {
        o.posI_src[l] = posI[enr0[l]];
        o.posG_src[l] = posG[enr0[l]];
        if (o.posI_src[l] >= 0) first[l] = std::min(first[l], o.posI_src[l]);
        if (o.posI_sink >= 0) first[l] = std::min(first[l], o.posI_sink);
    }
    o.first = first;
    o.gsort.resize(o.m);
    std::iota(o.gsort.begin(), o.gsort.end(), 0);
    std::stable_sort(o.gsort.begin(), o.gsort.end(), [&](int a, int b) { return first[o.L + a] < first[o.L + b]; });
    o.gfirst.resize(o.m);
    for (int q = 0; q < o.m; ++q) o.gfirst[q] = first[o.L + o.gsort[q]];
    // columns by their first non-zero row, so that a block's forward pass
    // starts where its earliest column does
    const int ncol = o.L + o.m;
    o.col_order.resize(ncol);
    std::iota(o.col_order.begin(), o.col_order.end(), 0);
    std::stable_sort(o.col_order.begin(), o.col_order.end(), [&](int a, int b) { return first[a] < first[b]; });
    for (int b0 = 0; b0 < ncol; b0 += R) {
        const int f = first[o.col_order[b0]];
        o.blk_start.push_back(f >= o.nI ? o.nI : f / SCHUR_MS_BB * SCHUR_MS_BB);
    }
    return CRT_OK;
}

namespace {

template <typename T> __device__ __forceinline__ T shfl_w(T v, int src, int width);
template <> __device__ __forceinline__ double shfl_w<double>(double v, int src, int width)
{
    return __shfl_sync(0xffffffffu, v, src, width);
}
template <> __device__ __forceinline__ cd shfl_w<cd>(cd v, int src, int width)
{
    return cd{__shfl_sync(0xffffffffu, v.x, src, width), __shfl_sync(0xffffffffu, v.y, src, width)};
}
// acc += a b (complex: four fused multiply-adds)
__device__ __forceinline__ void fma_acc(cd& acc, cd a, cd b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void fma_acc(double& acc, double a, double b) { acc = fma(a, b, acc); }

template <typename T> __device__ __forceinline__ T shfl_xor_t(T v, int mask);
template <> __device__ __forceinline__ double shfl_xor_t<double>(double v, int mask)
{
    return __shfl_xor_sync(0xffffffffu, v, mask);
}
template <> __device__ __forceinline__ cd shfl_xor_t<cd>(cd v, int mask)
{
    return cd{__shfl_xor_sync(0xffffffffu, v.x, mask), __shfl_xor_sync(0xffffffffu, v.y, mask)};
}

// one element global -> shared, asynchronously (cp.async; both addresses
// aligned to the element)
template <typename T> __device__ __forceinline__ void cp_async_elem(T* dst, const T* src);
template <> __device__ __forceinline__ void cp_async_elem<cd>(cd* dst, const cd* src) { cp_async16(dst, src); }
template <> __device__ __forceinline__ void cp_async_elem<double>(double* dst, const double* src)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}

// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_schur_rhs_src(SchurArgs s, const double* __restrict__ fakws, T* X)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= s.K * s.L) return;
    const int k = idx / s.L, l = idx % s.L;
    T* col = X + ((size_t)k * s.ncol + l) * s.nI;
    const double* fk = fakws + (size_t)k * s.nI;
    // r = e_src - e_sink (A pot = r; the reference's b = -r, src/kompab.f90),
    // scaled by fak
    if (s.posI_src[l] >= 0) col[s.posI_src[l]] = scale(Sc<T>::one(), fk[s.posI_src[l]]);
    if (s.lsink && s.posI_sink >= 0) col[s.posI_sink] -= scale(Sc<T>::one(), fk[s.posI_sink]);
}

template <typename T>
__global__ void k_schur_rhs_cpl(SchurArgs s, BandArgs<T> A, const double* __restrict__ fakws, T* X, T* cval)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.K * s.ncpl) return;
    const int k = (int)(idx / s.ncpl), q = (int)(idx % s.ncpl);
    // an interior-boundary entry has area contributions only (l unused)
    const T a = band_assemble_entry<T>(A, s.gi_ent[q], k, 0);
    cval[idx] = a;
    const int i = s.gi_pos[q];
    X[((size_t)k * s.ncol + s.L + s.gi_g[q]) * s.nI + i] = scale(a, fakws[(size_t)k * s.nI + i]);
}

// Lrev[k][c'][d] = L(r, r - d), r = n - 1 - c' (0 where r - d < 0).
template <typename T>
__global__ void k_schur_transpose(SchurArgs s, const T* __restrict__ Lws, T* Lrev)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = s.nI, W = s.WI;
    const long long per = (long long)n * W;
    if (idx >= (long long)s.nk * per) return;
    const int k = s.k0 + (int)(idx / per), cp = (int)((idx % per) / W), d = (int)(idx % W);
    const int r = n - 1 - cp, c = r - d;
    const T* Lk = Lws + (size_t)k * per;
    Lrev[(size_t)k * per + idx % per] = (c >= 0 && d <= s.mbI) ? Lk[(size_t)c * W + d] : Sc<T>::zero();
}

// ---------------------------------------------------------------------------
// Banded lower-triangular sweep L z = b for R columns per CTA: grid (column
// blocks, K).  The factor's columns stream through shared memory BB at a
// time (one bulk copy each, double-buffered, bounded mbarrier wait); the
// right-hand sides live in a window Z[WZ][R] (row r at slot r mod WZ,
// WZ >= mb + 3 BB), their rows arriving by cp.async two blocks ahead of
// use.  Per block: the BB x BB triangle (one half-warp per column, shuffle
// broadcasts, lane t holding row t), the finished rows out, and the
// (mb x BB) x (BB x R) update of the rows below (4 x TC register tiles).
//   back == 0: forward sweep of X's columns (col_order, from each block's
//     first non-zero row), in place;
//   back == 1: the back sweep L^T x^ = z^ of the source columns: Lws holds
//     the reversed row-packed factor and the rows are read reversed; the
//     solution goes out as kpot = fak x^ at the interior rows' nodes.
template <typename T, int NT, int R, int BB, int TC = 4, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_schur_sweep(SchurArgs s, const T* __restrict__ Lws,
                                                          const double* __restrict__ fakws, T* X, cd* kpot, int n_kpot,
                                                          int WZ, int back, int ahead = 2)
{
    static_assert(BB == 16 && R % 4 == 0 && R <= 32 && NT % 32 == 0 && NT >= R && (TC == 4 || TC == 2),
                  "sweep layout");
    extern __shared__ __align__(16) unsigned char sw_dyn[];
    const int W = s.WI, n = s.nI, mb = s.mbI;
    T* Lb = reinterpret_cast<T*>(sw_dyn);   // [2][BB * W]
    T* Z = Lb + 2 * BB * W;                 // [WZ][R]
    __shared__ T dinv[BB];
    __shared__ int colid[R];
    __shared__ __align__(8) unsigned long long bar[2];
    __shared__ int s_err;
    const int tid = threadIdx.x;
    // wavenumbers along x: the CTAs start in the order of their blocks'
    // first rows, longest passes first over all wavenumbers
    const int blk = blockIdx.y, k = s.k0 + blockIdx.x;
    const int start = back ? 0 : s.blk_start[blk];
    if (start >= n) return;   // every column of the block is zero, and so is its solution
    const T* Lk = Lws + (size_t)k * n * W;
    if (tid < R) {
        const int c = blk * R + tid;
        colid[tid] = back ? (c < s.L ? c : -1) : (c < s.ncol ? s.col_order[c] : -1);
    }
    if (tid == 0) {
        s_err = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    __syncthreads();
    int ph0 = 0, ph1 = 0;
    auto colp = [&](int j) { return X + ((size_t)k * s.ncol + colid[j]) * n; };
    auto fetch = [&](int c0, int buf) {
        if (tid == 0) {
            if (s.progress && !s_err) {
                // the factor's columns [c0, c0 + BB) are final once its
                // progress passes them.  The wait gives up after about 4 s,
                // or at once when another CTA of this wavenumber gave up
                // (status set); the result is then flagged as failed.
                const int want = min(n, c0 + BB);
                long polls = 0;
                int got;
                while (true) {
                    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(got) : "l"(s.progress + k) : "memory");
                    if (got >= want) break;
                    if (*(volatile const int*)(s.status + k) != 0 || ++polls > (1L << 22)) {
                        s_err = 1;
                        atomicMax(&s.status[k], (int)CRT_ERR_CUDA);
                        break;
                    }
                    __nanosleep(256);
                }
                // the copy below reads them through the async proxy
                asm volatile("fence.proxy.async.global;\n" ::: "memory");
            }
            const int bytes = min(BB, n - c0) * W * (int)sizeof(T);
            mbar_expect_tx(&bar[buf], bytes);
            bulk_g2s(Lb + (size_t)buf * BB * W, Lk + (size_t)c0 * W, bytes, &bar[buf]);
        }
    };
    auto wait = [&](int buf) {
        int& ph = buf ? ph1 : ph0;
        if (!mbar_wait(&bar[buf], ph)) s_err = 1;
        ph ^= 1;
    };
    // rows [r0, r1) of every column into their slots, one commit group
    auto issue_rows = [&](int r0, int r1) {
        const int nr = r1 - r0;
        for (int idx = tid; idx < nr * R; idx += NT) {
            const int j = idx / nr, r = r0 + idx % nr;
            T* dst = Z + (size_t)(r % WZ) * R + j;
            if (colid[j] >= 0) cp_async_elem<T>(dst, colp(j) + (back ? n - 1 - r : r));
            else *dst = Sc<T>::zero();
        }
        cp_async_commit();
    };
    // rows arrive `ahead` blocks before use: 2 (WZ >= mb + 3 BB, the wait at
    // the end of a block leaves one group in flight) or 1 (WZ >= mb + 2 BB,
    // the rows issued at the start of a block awaited at its end: the
    // smaller window lets two CTAs share an SM)
    issue_rows(start, min(n, start + BB + mb));
    if (ahead == 2) issue_rows(min(n, start + BB + mb), min(n, start + 2 * BB + mb));
    fetch(start, 0);
    if (ahead == 2) cp_async_wait_group<1>();
    else cp_async_wait_group<0>();
    __syncthreads();
    int buf = 0;
    for (int c0 = start; c0 < n; c0 += BB) {
        const int nb = min(BB, n - c0);
        wait(buf);
        if (c0 + BB < n) fetch(c0 + BB, buf ^ 1);
        // the rows `ahead` blocks ahead (their slots held rows finished a block ago)
        issue_rows(min(n, c0 + (ahead + 1) * BB + mb - BB), min(n, c0 + (ahead + 1) * BB + mb));
        const T* Lc = Lb + (size_t)buf * BB * W;
        if (tid < nb) dinv[tid] = Sc<T>::recip(Lc[tid * W]);
        __syncthreads();
        // the block's rows sit in consecutive slots (WZ is a multiple of BB)
        const int sb = c0 % WZ;
        {   // the block's triangle: a half-warp per column, lane t holds row t
            // and its row of the block's L in registers; at step u lane u
            // finishes its row and hands it to the half-warp by a shuffle, so
            // every row takes z_t -= L_tu z_u for u = 0 .. t-1, then z_t *= 1/L_tt
            constexpr int HW = NT / 16;   // half-warps of the CTA (NT is a multiple of 32)
            const int hw = tid >> 4, lt = tid & 15;
            for (int j0 = 0; j0 < R; j0 += HW) {
                const int j = j0 + hw;
                const bool act = j < R && lt < nb;
                T zt = Sc<T>::zero(), lrow[BB];
#pragma unroll
                for (int u = 0; u < BB; ++u)
                    lrow[u] = (act && u < lt && lt - u <= mb) ? Lc[u * W + (lt - u)] : Sc<T>::zero();
                if (act) zt = Z[(size_t)(sb + lt) * R + j];
#pragma unroll
                for (int u = 0; u < BB; ++u) {
                    if (u < nb) {
                        if (lt == u) zt = Sc<T>::mul(zt, dinv[u]);
                        const T zu = shfl_w<T>(zt, u, 16);
                        if (lt > u && lt < nb && lt - u <= mb) fms_acc(zt, lrow[u], zu);
                    }
                }
                if (act) Z[(size_t)(sb + lt) * R + j] = zt;
            }
        }
        __syncthreads();
        // the block's rows are final: out
        for (int idx = tid; idx < nb * R; idx += NT) {
            const int j = idx / nb, t = idx % nb;
            if (colid[j] < 0) continue;
            const int r = c0 + t;
            const T v = Z[(size_t)(sb + t) * R + j];
            if (!back) {
                colp(j)[r] = v;
            } else {
                const int i = n - 1 - r;
                kpot[((size_t)k * s.L + colid[j]) * n_kpot + s.permI[i]] =
                    Sc<T>::to_cd(scale(v, fakws[(size_t)k * n + i]));
            }
        }
        {   // rows [c0 + nb, c0 + nb + mb) take the block's columns: a thread
            // owns rows rq + NQ a (4 of them) and columns jq + (R/TC) c (TC of
            // them), so a warp's loads fall on consecutive words; every entry
            // takes the block's columns u = 0 .. nb-1 in order, whatever TC
            const int rlo = c0 + nb, rhi = min(n, c0 + nb + mb);
            const int NQ = (rhi - rlo + 3) >> 2;
            constexpr int RJ = R / TC;
            for (int tile = tid; tile < NQ * RJ; tile += NT) {
                const int rq = tile / RJ, jq = tile % RJ;
                T acc[4][TC];
                int sl[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int r = rlo + rq + NQ * a;
                    sl[a] = r < rhi ? r % WZ : -1;
#pragma unroll
                    for (int c = 0; c < TC; ++c)
                        acc[a][c] = sl[a] >= 0 ? Z[(size_t)sl[a] * R + jq + RJ * c] : Sc<T>::zero();
                }
#pragma unroll
                for (int u = 0; u < BB; ++u) {
                    if (u < nb) {
                        T zc[TC], lv[4];
#pragma unroll
                        for (int c = 0; c < TC; ++c) zc[c] = Z[(size_t)(sb + u) * R + jq + RJ * c];
#pragma unroll
                        for (int a = 0; a < 4; ++a) {
                            const int d = rlo + rq + NQ * a - (c0 + u);
                            lv[a] = (sl[a] >= 0 && d <= mb) ? Lc[u * W + d] : Sc<T>::zero();
                        }
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int c = 0; c < TC; ++c) fms_acc(acc[a][c], lv[a], zc[c]);
                    }
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    if (sl[a] >= 0)
#pragma unroll
                        for (int c = 0; c < TC; ++c) Z[(size_t)sl[a] * R + jq + RJ * c] = acc[a][c];
            }
        }
        // the buffer just read is the destination of the bulk copy after next
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if (ahead == 2) cp_async_wait_group<1>();   // the rows of the next block have landed
        else cp_async_wait_group<0>();
        __syncthreads();
        buf ^= 1;
    }
    cp_async_wait_group<0>();
    if (tid == 0 && s_err) atomicMax(&s.status[k], (int)CRT_ERR_CUDA);
}

// ---------------------------------------------------------------------------
// The sweeps with R = 16 columns per CTA (512 threads) and the triangle
// beside the update (back: the source columns of the back sweep; forward:
// the 16-column blocks of the forward sweep, CRT_B200_SCHUR_R=16): per block b (rows c0 .. c0 + 16), between
// barriers,
//   A. warps 0-7 solve block b's triangle (a half-warp per column, lane t
//      holding row t; the finished row handed on by a shuffle) while warps
//      8-15 take block b-1's columns into the rows past block b (those of
//      block b took them in phase B of block b-1);
//   B. threads 0-255 take block b's columns into block b+1's rows (an entry
//      each) while warps 8-15 write block b's rows out.
// Every row takes the blocks' columns in block order and each block's
// columns in order, with the operations of k_schur_sweep; the factor's
// column blocks b-1, b, b+1 sit in three buffers.
template <typename T>
__global__ void __launch_bounds__(512, 1) k_schur_sweep_pp(SchurArgs s, const T* __restrict__ Lws,
                                                         const double* __restrict__ fakws, T* X, cd* kpot,
                                                         int n_kpot, int WZ, int back)
{
    constexpr int R = 16, BB = 16, NT = 512, TC = 2;
    extern __shared__ __align__(16) unsigned char bp_dyn[];
    const int W = s.WI, n = s.nI, mb = s.mbI;
    T* Lb = reinterpret_cast<T*>(bp_dyn);   // [3][BB * W]
    T* Z = Lb + 3 * BB * W;                 // [WZ][R]
    __shared__ T dinv[BB];
    __shared__ int colid[R];
    __shared__ __align__(8) unsigned long long bar[3];
    __shared__ int s_err;
    const int tid = threadIdx.x;
    const int blk = blockIdx.y, k = s.k0 + blockIdx.x;
    const int start = back ? 0 : s.blk_start[blk];
    if (start >= n) return;   // every column of the block is zero, and so is its solution
    const T* Lk = Lws + (size_t)k * n * W;
    if (tid < R) {
        const int c = blk * R + tid;
        colid[tid] = back ? (c < s.L ? c : -1) : (c < s.ncol ? s.col_order[c] : -1);
    }
    if (tid == 0) {
        s_err = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&bar[2], 1);
    }
    __syncthreads();
    int phs = 0;
    auto fetch = [&](int c0, int buf) {
        if (tid == 0) {
            if (s.progress && !s_err) {
                // beside the factor: its columns [c0, c0 + BB) are final once
                // its progress passes them (bounded wait, as k_schur_sweep)
                const int want = min(n, c0 + BB);
                long polls = 0;
                int got;
                while (true) {
                    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(got) : "l"(s.progress + k) : "memory");
                    if (got >= want) break;
                    if (*(volatile const int*)(s.status + k) != 0 || ++polls > (1L << 22)) {
                        s_err = 1;
                        atomicMax(&s.status[k], (int)CRT_ERR_CUDA);
                        break;
                    }
                    __nanosleep(256);
                }
                asm volatile("fence.proxy.async.global;\n" ::: "memory");
            }
            const int bytes = min(BB, n - c0) * W * (int)sizeof(T);
            mbar_expect_tx(&bar[buf], bytes);
            bulk_g2s(Lb + (size_t)buf * BB * W, Lk + (size_t)c0 * W, bytes, &bar[buf]);
        }
    };
    auto wait = [&](int buf) {
        if (!mbar_wait(&bar[buf], (phs >> buf) & 1)) s_err = 1;
        phs ^= 1 << buf;
    };
    auto colp = [&](int j) { return X + ((size_t)k * s.ncol + colid[j]) * n; };   // the column's rows in X
    auto issue_rows = [&](int r0, int r1) {
        const int nr = r1 - r0;
        for (int idx = tid; idx < nr * R; idx += NT) {
            const int j = idx / nr, r = r0 + idx % nr;
            T* dst = Z + (size_t)(r % WZ) * R + j;
            if (colid[j] >= 0) cp_async_elem<T>(dst, colp(j) + (back ? n - 1 - r : r));
            else *dst = Sc<T>::zero();
        }
        cp_async_commit();
    };
    // rows [rlo, rhi) take the columns of the block at cb (nbb rows, factor
    // block Lq), threads [t0, t0 + nt): 4 rows x TC columns per thread
    auto update_rows = [&](const T* Lq, int cb, int nbb, int rlo, int rhi, int t0, int nt) {
        if (rlo >= rhi) return;
        const int NQ = (rhi - rlo + 3) >> 2;
        constexpr int RJ = R / TC;
        const int sbb = cb % WZ;
        for (int tile = tid - t0; tile < NQ * RJ; tile += nt) {
            const int rq = tile / RJ, jq = tile % RJ;
            T acc[4][TC];
            int sl[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int r = rlo + rq + NQ * a;
                sl[a] = r < rhi ? r % WZ : -1;
#pragma unroll
                for (int c = 0; c < TC; ++c)
                    acc[a][c] = sl[a] >= 0 ? Z[(size_t)sl[a] * R + jq + RJ * c] : Sc<T>::zero();
            }
#pragma unroll
            for (int u = 0; u < BB; ++u) {
                if (u < nbb) {
                    T zc[TC], lv[4];
#pragma unroll
                    for (int c = 0; c < TC; ++c) zc[c] = Z[(size_t)(sbb + u) * R + jq + RJ * c];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int d = rlo + rq + NQ * a - (cb + u);
                        lv[a] = (sl[a] >= 0 && d <= mb) ? Lq[u * W + d] : Sc<T>::zero();
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < TC; ++c) fms_acc(acc[a][c], lv[a], zc[c]);
                }
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
                if (sl[a] >= 0)
#pragma unroll
                    for (int c = 0; c < TC; ++c) Z[(size_t)sl[a] * R + jq + RJ * c] = acc[a][c];
        }
    };
    issue_rows(start, min(n, start + BB + mb));
    issue_rows(min(n, start + BB + mb), min(n, start + 2 * BB + mb));
    fetch(start, 0);
    if (start + BB < n) fetch(start + BB, 1);
    cp_async_wait_group<1>();
    __syncthreads();
    int bi = 0;
    for (int c0 = start; c0 < n; c0 += BB, ++bi) {
        const int nb = min(BB, n - c0);
        const int cur = bi % 3, prv = (bi + 2) % 3;
        wait(cur);
        const T* Lc = Lb + (size_t)cur * BB * W;
        const T* Lp = Lb + (size_t)prv * BB * W;
        if (tid < nb) dinv[tid] = Sc<T>::recip(Lc[tid * W]);
        __syncthreads();
        const int sb = c0 % WZ;
        if (tid < 256) {
            // A. block b's triangle: half-warp hw = column, lane lt = row
            const int j = tid >> 4, lt = tid & 15;
            const bool act = lt < nb;
            T zt = Sc<T>::zero(), lrow[BB];
#pragma unroll
            for (int u = 0; u < BB; ++u)
                lrow[u] = (act && u < lt && lt - u <= mb) ? Lc[u * W + (lt - u)] : Sc<T>::zero();
            if (act) zt = Z[(size_t)(sb + lt) * R + j];
#pragma unroll
            for (int u = 0; u < BB; ++u) {
                if (u < nb) {
                    if (lt == u) zt = Sc<T>::mul(zt, dinv[u]);
                    const T zu = shfl_w<T>(zt, u, 16);
                    if (lt > u && lt < nb && lt - u <= mb) fms_acc(zt, lrow[u], zu);
                }
            }
            if (act) Z[(size_t)(sb + lt) * R + j] = zt;
        } else if (c0 > start) {
            // A. block b-1 (BB rows) into rows [c0 + BB, c0 + mb)
            update_rows(Lp, c0 - BB, BB, min(n, c0 + BB), min(n, c0 + mb), 256, 256);
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid < 256) {
            // B. block b's columns into block b+1's rows, an entry (row, column) per thread
            const int j = tid & 15, t = tid >> 4, r = c0 + nb + t;
            if (r < n && t < BB) {
                T z = Z[(size_t)(r % WZ) * R + j];
#pragma unroll
                for (int u = 0; u < BB; ++u) {
                    const int d = r - (c0 + u);
                    if (u < nb && d <= mb) fms_acc(z, Lc[u * W + d], Z[(size_t)(sb + u) * R + j]);
                }
                Z[(size_t)(r % WZ) * R + j] = z;
            }
        } else {
            // B. block b's rows out
            for (int idx = tid - 256; idx < nb * R; idx += 256) {
                const int jj = idx / nb, t = idx % nb;
                if (colid[jj] < 0) continue;
                const int r = c0 + t;
                const T v = Z[(size_t)(sb + t) * R + jj];
                if (!back) {
                    colp(jj)[r] = v;
                } else {
                    const int i = n - 1 - r;
                    kpot[((size_t)k * s.L + colid[jj]) * n_kpot + s.permI[i]] =
                        Sc<T>::to_cd(scale(v, fakws[(size_t)k * n + i]));
                }
            }
        }
        if (c0 + 2 * BB < n) fetch(c0 + 2 * BB, prv);
        issue_rows(min(n, c0 + 2 * BB + mb), min(n, c0 + 3 * BB + mb));
        cp_async_wait_group<1>();
        __syncthreads();
    }
    cp_async_wait_group<0>();
    if (tid == 0 && s_err) atomicMax(&s.status[k], (int)CRT_ERR_CUDA);
}

// ---------------------------------------------------------------------------
// C[k][c][g] = sum_i V^[i][g] X[i][c] over the rows where both columns can
// be non-zero; tiles 64 (g) x 32 (c), 128 threads of 4 x 4.  The tiles of
// the V^T V^ block above its diagonal are skipped (the Cholesky reads the
// lower triangle).
template <typename T>
__global__ void __launch_bounds__(128) k_schur_gram(SchurArgs s, const T* __restrict__ X, T* C)
{
    constexpr int TG = 64, TC = 32, TI = 16;
    extern __shared__ __align__(16) unsigned char gram_dyn[];   // both stages of both tiles
    auto As = reinterpret_cast<T(*)[TI][TG + 1]>(gram_dyn);                                  // [2][TI][TG + 1]
    auto Bs = reinterpret_cast<T(*)[TI][TC + 1]>(gram_dyn + 2 * TI * (TG + 1) * sizeof(T));  // [2][TI][TC + 1]
    __shared__ int s_i0;
    // wavenumbers along x, so the long tiles (early first rows) of every
    // wavenumber start first
    const int tid = threadIdx.x, k = s.k0 + blockIdx.x;
    const int g0 = blockIdx.y * TG, c0 = blockIdx.z * TC;
    const int m = s.m, L = s.L, nI = s.nI, ncol = s.ncol;
    if (c0 >= L && c0 - L > g0 + TG - 1) return;
    if (tid == 0) {
        int fg = nI, fc = nI;
        for (int q = 0; q < TG && g0 + q < m; ++q) fg = min(fg, s.first[L + g0 + q]);
        for (int q = 0; q < TC && c0 + q < ncol; ++q) fc = min(fc, s.first[c0 + q]);
        s_i0 = max(fg, fc) / TI * TI;
    }
    __syncthreads();
    const int ti = tid % 16, tc = tid / 16;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = Sc<T>::zero();
    const T* Xk = X + (size_t)k * ncol * nI;
    // the tiles of rows [i0, i0 + TI) into buffer `buf` (cp.async, the
    // next block's copies in flight while this one is multiplied)
    auto stage = [&](int buf, int i0) {
        for (int idx = tid; idx < TI * TG; idx += 128) {
            const int gg = idx / TI, ii = idx % TI;
            if (g0 + gg < m && i0 + ii < nI) cp_async_elem<T>(&As[buf][ii][gg], Xk + (size_t)(L + g0 + gg) * nI + i0 + ii);
            else As[buf][ii][gg] = Sc<T>::zero();
        }
        for (int idx = tid; idx < TI * TC; idx += 128) {
            const int cc = idx / TI, ii = idx % TI;
            if (c0 + cc < ncol && i0 + ii < nI) cp_async_elem<T>(&Bs[buf][ii][cc], Xk + (size_t)(c0 + cc) * nI + i0 + ii);
            else Bs[buf][ii][cc] = Sc<T>::zero();
        }
        cp_async_commit();
    };
    int buf = 0;
    if (s_i0 < nI) stage(0, s_i0);
    for (int i0 = s_i0; i0 < nI; i0 += TI, buf ^= 1) {
        if (i0 + TI < nI) {
            stage(buf ^ 1, i0 + TI);   // its last readers finished before the trailing barrier
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();
#pragma unroll 4
        for (int ii = 0; ii < TI; ++ii) {
            T a4[4], b4[4];
            // rows ti + 16 a, columns tc + 8 c: a warp reads consecutive words
#pragma unroll
            for (int a = 0; a < 4; ++a) a4[a] = As[buf][ii][ti + 16 * a];
#pragma unroll
            for (int c = 0; c < 4; ++c) b4[c] = Bs[buf][ii][tc + 8 * c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) fma_acc(acc[a][c], a4[a], b4[c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int cc = c0 + tc + 8 * c;
        if (cc >= ncol) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int g = g0 + ti + 16 * a;
            if (g < m) C[((size_t)k * ncol + cc) * m + g] = acc[a][c];
        }
    }
}

// ---------------------------------------------------------------------------
// Dense Cholesky of the Schur complements, one CTA per (k, l) system:
// S = A_GG(l) - C_VV (lower triangle, column-major, in the workspace),
// right-looking with an NB-column panel in shared memory; the forward solve
// L y = r_G - C[l] rides along each column, the back solve L^T x = y goes
// panel by panel from the last (dot products of the panel columns, then the
// panel's triangle on one warp).
//
// PF: the next super-tile's entries are loaded into registers while the
// current one is updated (one CTA per SM); without, two CTAs share an SM and
// hide each other's latency.
// REF: the reference factors of the iterative form instead, one per
// (wavenumber, electrode group) b: S0 + the group's mean mixed-boundary part
// (S0 from C), factored in place without a right-hand side; a non-positive
// pivot is counted in *nonconv.
template <typename T, int NT, int NB, bool PF, bool REF = false>
__global__ void __launch_bounds__(NT, PF ? 1 : 2) k_schur_chol(SchurArgs s, BandArgs<T> A, const T* __restrict__ C,
                                                               T* Sws, T* xg, int sys0, int* nonconv = nullptr)
{
    static_assert(NT == 256 && NB <= 16, "chol layout");
    extern __shared__ __align__(16) unsigned char ch_dyn[];
    const int m = s.m;
    T* P = reinterpret_cast<T*>(ch_dyn);   // panel [NB][m]: P[t m + r] = L(r, p0 + t)
    T* y = P + (size_t)NB * m;             // [m]
    __shared__ int s_err;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x, sys = sys0 + b;
    const int k = REF ? b / s.ngrp : sys / s.L, l = REF ? (b % s.ngrp) * s.grp : sys % s.L;
    T* S = Sws + (size_t)b * m * m;
    const T* Ck = C + (size_t)k * s.ncol * m;
    if (tid == 0) s_err = 0;
    if constexpr (REF) {
        const T* S0k = C;   // REF: C is S0 ([k][m][m], both triangles)
        for (int c = 0; c < m; ++c)
            for (int r = c + tid; r < m; r += NT) S[(size_t)c * m + r] = S0k[((size_t)k * m + c) * m + r];
        for (int g = tid; g < m; g += NT) y[g] = Sc<T>::zero();
        __syncthreads();
        const int nl = min(s.grp, s.L - l);
        for (int g = tid; g < m; g += NT)
            for (int q = s.bd_ptr[g]; q < s.bd_ptr[g + 1]; ++q) {
                const int h = s.bd_col[q];
                if (h <= g) S[(size_t)h * m + g] += band_assemble_part<T>(A, s.bd_ent[q], k, l, nl, 1);
            }
    } else {
        for (int c = 0; c < m; ++c) {
            const T* src = Ck + (size_t)(s.L + c) * m;
            for (int r = c + tid; r < m; r += NT) S[(size_t)c * m + r] = -src[r];
        }
        for (int g = tid; g < m; g += NT) {
            T v = -Ck[(size_t)l * m + g];
            if (g == s.posG_src[l]) v += Sc<T>::one();
            if (s.lsink && g == s.posG_sink) v -= Sc<T>::one();
            y[g] = v;
        }
        __syncthreads();
        for (int q = tid; q < s.ngg; q += NT) {
            const T a = band_assemble_entry<T>(A, s.gg_ent[q], k, l);
            S[(size_t)s.gg_h[q] * m + s.gg_g[q]] += a;
        }
    }
    __syncthreads();
    for (int p0 = 0; p0 < m; p0 += NB) {
        const int nb = min(NB, m - p0);
        for (int t = 0; t < nb; ++t)
            for (int r = p0 + tid; r < m; r += NT) P[t * m + r] = S[(size_t)(p0 + t) * m + r];
        __syncthreads();
        for (int t = 0; t < nb; ++t) {
            const int c = p0 + t;
            const T piv = P[t * m + c];
            if (Sc<T>::bad_pivot(piv)) s_err = CRT_ERR_PIVOT;
            T root, inv;
            Sc<T>::sqrt_recip(piv, root, inv);
            const T yc = Sc<T>::mul(y[c], inv);
            __syncthreads();   // every thread has read the pivot and y[c]
            for (int r = c + 1 + tid; r < m; r += NT) {
                const T lv = Sc<T>::mul(P[t * m + r], inv);
                P[t * m + r] = lv;
                fms_acc(y[r], lv, yc);
            }
            if (tid == 0) {
                P[t * m + c] = root;
                y[c] = yc;
            }
            __syncthreads();
            const int rows = m - c - 1;
            for (int idx = tid; idx < (nb - t - 1) * rows; idx += NT) {
                const int tt = t + 1 + idx / rows, r = c + 1 + idx % rows;
                if (r >= p0 + tt) fms_acc(P[tt * m + r], P[t * m + r], P[t * m + p0 + tt]);
            }
            __syncthreads();
        }
        if (s_err) break;
        for (int t = 0; t < nb; ++t)
            for (int r = p0 + t + tid; r < m; r += NT) S[(size_t)(p0 + t) * m + r] = P[t * m + r];
        // trailing update of the lower triangle below the panel by 64 x 64
        // super-tiles (their lower triangle on the diagonal): thread (ti, tj)
        // owns rows ti + 16 a and columns tj + 16 c of each, so a warp's
        // loads of S are two 256-byte runs and its panel reads consecutive
        // words; the next super-tile's entries load while the current one
        // is updated
        const int q0 = p0 + nb, mt = m - q0;
        if (mt > 0) {
            const int NS = (mt + 63) / 64, nst = NS * (NS + 1) / 2;
            const int ti = tid & 15, tj = tid >> 4;
            auto st_origin = [&](int st, int& R0, int& C0) {
                int SX = (int)((sqrtf(8.0f * st + 1.0f) - 1.0f) * 0.5f);
                while ((SX + 1) * (SX + 2) / 2 <= st) ++SX;
                while (SX * (SX + 1) / 2 > st) --SX;
                R0 = q0 + 64 * SX;
                C0 = q0 + 64 * (st - SX * (SX + 1) / 2);
            };
            auto st_load = [&](int st, T (&v)[4][4]) {
                int R0, C0;
                st_origin(st, R0, C0);
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int r = R0 + ti + 16 * a, cc = C0 + tj + 16 * c;
                        v[a][c] = (r < m && cc < m && r >= cc) ? S[(size_t)cc * m + r] : Sc<T>::zero();
                    }
            };
            T cur[4][4], nxt[4][4];
            st_load(0, cur);
            for (int st = 0; st < nst; ++st) {
                if (PF && st + 1 < nst) st_load(st + 1, nxt);
                int R0, C0;
                st_origin(st, R0, C0);
                for (int t = 0; t < nb; ++t) {
                    T pr[4], pc[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int r = R0 + ti + 16 * a, cc = C0 + tj + 16 * a;
                        pr[a] = r < m ? P[t * m + r] : Sc<T>::zero();
                        pc[a] = cc < m ? P[t * m + cc] : Sc<T>::zero();
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < 4; ++c) fms_acc(cur[a][c], pr[a], pc[c]);
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int r = R0 + ti + 16 * a, cc = C0 + tj + 16 * c;
                        if (r < m && cc < m && r >= cc) S[(size_t)cc * m + r] = cur[a][c];
                        if (PF) cur[a][c] = nxt[a][c];
                    }
                if (!PF && st + 1 < nst) st_load(st + 1, cur);
            }
        }
        __syncthreads();
    }
    if constexpr (REF) {
        if (s_err && tid == 0) atomicAdd(nonconv, 1);
        return;
    }
    if (s_err) {
        if (tid == 0) atomicMax(&s.status[sys], s_err);
        return;
    }
    // L^T x = y, panel by panel from the last
    for (int p0 = (m - 1) / NB * NB; p0 >= 0; p0 -= NB) {
        const int nb = min(NB, m - p0);
        for (int t = 0; t < nb; ++t)
            for (int r = p0 + tid; r < m; r += NT) P[t * m + r] = S[(size_t)(p0 + t) * m + r];
        __syncthreads();
        {   // y[p0 + t] -= sum over solved rows r >= p0 + nb of L(r, p0 + t) x_r
            const int t = tid >> 4, sl = tid & 15;
            T part = Sc<T>::zero();
            if (t < nb)
                for (int r = p0 + nb + sl; r < m; r += 16) fma_acc(part, P[t * m + r], y[r]);
#pragma unroll
            for (int off = 8; off > 0; off >>= 1) part += shfl_xor_t(part, off);
            if (sl == 0 && t < nb) y[p0 + t] -= part;
        }
        __syncthreads();
        if (warp == 0) {   // the panel's triangle of L^T, lane t = row p0 + t
            T v = lane < nb ? y[p0 + lane] : Sc<T>::zero();
            for (int u = nb - 1; u >= 0; --u) {
                if (lane == u) v = Sc<T>::mul(v, Sc<T>::recip(P[u * m + p0 + u]));
                const T x = shfl_w(v, u, 32);
                if (lane < u) fms_acc(v, P[lane * m + p0 + u], x);
            }
            if (lane < nb) y[p0 + lane] = v;
        }
        __syncthreads();
    }
    for (int g = tid; g < m; g += NT) xg[(size_t)sys * m + g] = y[g];
}

// |Re| + |Im| (the convergence test's magnitude)
__device__ __forceinline__ double mag1(double a) { return fabs(a); }
__device__ __forceinline__ double mag1(cd a) { return fabs(a.x) + fabs(a.y); }

// ---------------------------------------------------------------------------
// Iterative form.  S0[k] = A_GG^area - V^T V^, both triangles, column-major:
// first -C_VV (C's lower triangle, mirrored), then the area part of every G-G
// entry (each pair g >= h occurs once in the gg list).
template <typename T>
__global__ void k_schur_s0_vv(SchurArgs s, const T* __restrict__ C, T* S0)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = s.m;
    if (idx >= (long long)s.K * m * m) return;
    const int k = (int)(idx / ((long long)m * m)), c = (int)((idx / m) % m), r = (int)(idx % m);
    const int hi = max(r, c), lo = min(r, c);
    S0[idx] = -C[((size_t)k * s.ncol + s.L + lo) * m + hi];
}

template <typename T>
__global__ void k_schur_s0_area(SchurArgs s, BandArgs<T> A, T* S0)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.K * s.ngg) return;
    const int k = (int)(idx / s.ngg), q = (int)(idx % s.ngg), m = s.m;
    const T a = band_assemble_part<T>(A, s.gg_ent[q], k, 0, 1, 0);
    const int g = s.gg_g[q], h = s.gg_h[q];
    T* Sk = S0 + (size_t)k * m * m;
    Sk[(size_t)h * m + g] += a;
    if (g != h) Sk[(size_t)g * m + h] += a;
}

// The preconditioned iteration for NS systems of one electrode group (one
// CTA): x_0 = 0, r = b - S_l x, z = S_ref^-1 r, x += z, until
// max |z| <= tol max |x| for every system.  X and R/Z live in shared memory,
// a system's column contiguous ([NS][m], so that threads over rows touch
// consecutive words); S0 and the reference factor stream from L2.  The
// products S0 X read S0 by columns (coalesced over the rows); D_l X uses the
// boundary rows (bd_*); the triangular solves go by 16-column panels (one
// warp per system solves a panel's triangle, all threads update the rows
// below, or, backwards, reduce the solved rows into the panel).
constexpr int SCHUR_IT_NS = 8;
constexpr int SCHUR_IT_NT = 256;
constexpr int SCHUR_IT_PB = 16;

template <typename T>
__global__ void k_schur_dvals(SchurArgs s, BandArgs<T> A, T* Dv)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.K * s.L * s.nbd) return;
    const int q = (int)(idx % s.nbd);
    const long long kl = idx / s.nbd;
    const int k = (int)(kl / s.L), l = (int)(kl % s.L);
    Dv[idx] = band_assemble_part<T>(A, s.bd_ent[q], k, l, 1, 1);
}

// NS systems per CTA (8, or 4 at two CTAs per SM: MINB); each system's
// arithmetic does not depend on NS.
template <typename T, int NS = SCHUR_IT_NS, int MINB = 1>
__global__ void __launch_bounds__(SCHUR_IT_NT, MINB) k_schur_iter(SchurArgs s, BandArgs<T> A, const T* __restrict__ C,
                                                                 const T* __restrict__ S0, const T* __restrict__ Lref,
                                                                 const T* __restrict__ Dv, T* xg, int maxit,
                                                                 double tol, int* nonconv)
{
    constexpr int NT = SCHUR_IT_NT, PB = SCHUR_IT_PB;
    extern __shared__ __align__(16) unsigned char it_dyn[];
    const int m = s.m, L = s.L;
    T* X = reinterpret_cast<T*>(it_dyn);   // [NS][m]: system j's column at j m
    T* Z = X + (size_t)m * NS;              // [NS][m]
    __shared__ double s_dx[NS], s_x[NS], s_dprev[NS];
    __shared__ int s_go;
    __shared__ T Ld[PB][PB + 1];   // the panel's diagonal block, Ld[c][r] = L(p0 + r, p0 + c)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cpg = (s.grp + NS - 1) / NS;             // CTAs per group
    const int b = blockIdx.x, half = b % cpg, kg = b / cpg, g = kg % s.ngrp, k = kg / s.ngrp;
    const int l0 = g * s.grp + half * NS;
    const int l1 = min(min(L, (g + 1) * s.grp), l0 + NS);
    const int ns = l1 - l0;
    if (ns <= 0) return;
    const T* Ck = C + (size_t)k * s.ncol * m;
    const T* Sk = S0 + (size_t)k * m * m;
    const T* Lg = Lref + (size_t)kg * m * m;
    auto bval = [&](int r, int j) {
        const int l = l0 + j;
        T v = -Ck[(size_t)l * m + r];
        if (r == s.posG_src[l]) v += Sc<T>::one();
        if (s.lsink && r == s.posG_sink) v -= Sc<T>::one();
        return v;
    };
    for (int i = tid; i < m * NS; i += NT) {
        const int j = i / m, r = i % m;
        X[i] = Sc<T>::zero();
        Z[i] = j < ns ? bval(r, j) : Sc<T>::zero();
    }
    __syncthreads();
    int it = 0;
    for (;; ++it) {
        if (it > 0) {
            // Z = b - S0 X - D_l X (rows r = tid, tid + NT, ...)
            for (int r = tid; r < m; r += NT) {
                T acc[NS];
#pragma unroll
                for (int j = 0; j < NS; ++j) acc[j] = j < ns ? bval(r, j) : Sc<T>::zero();
#pragma unroll 4
                for (int c = 0; c < m; ++c) {
                    const T a = Sk[(size_t)c * m + r];
#pragma unroll
                    for (int j = 0; j < NS; ++j) fms_acc(acc[j], a, X[j * m + c]);
                }
                const T* Dk = Dv + ((size_t)k * L + l0) * s.nbd;
                for (int q = s.bd_ptr[r]; q < s.bd_ptr[r + 1]; ++q) {
                    const int c = s.bd_col[q];
#pragma unroll
                    for (int j = 0; j < NS; ++j)
                        if (j < ns) fms_acc(acc[j], Dk[(size_t)j * s.nbd + q], X[j * m + c]);
                }
#pragma unroll
                for (int j = 0; j < NS; ++j) Z[j * m + r] = acc[j];
            }
            __syncthreads();
        }
        // the panel's diagonal block into shared memory (all threads)
        auto stage_diag = [&](int p0, int nb) {
            for (int i = tid; i < PB * PB; i += NT) {
                const int c = i / PB, r = i % PB;
                Ld[c][r] = (c < nb && r < nb && r >= c) ? Lg[(size_t)(p0 + c) * m + p0 + r] : Sc<T>::zero();
            }
        };
        // forward: L y = z, by panels
        for (int p0 = 0; p0 < m; p0 += PB) {
            const int nb = min(PB, m - p0);
            stage_diag(p0, nb);
            __syncthreads();
            if (warp < NS) {   // warp j: system j, lane t: row p0 + t
                const int j = warp;
                T v = lane < nb ? Z[j * m + p0 + lane] : Sc<T>::zero();
#pragma unroll
                for (int u = 0; u < PB; ++u) {
                    if (u < nb) {
                        if (lane == u) v = Sc<T>::mul(v, Sc<T>::recip(Ld[u][u]));
                        const T xu = shfl_w(v, u, 32);
                        if (lane > u && lane < nb) fms_acc(v, Ld[u][lane], xu);
                    }
                }
                if (lane < nb) Z[j * m + p0 + lane] = v;
            }
            __syncthreads();
            for (int r = p0 + nb + tid; r < m; r += NT) {
                T acc[NS];
#pragma unroll
                for (int j = 0; j < NS; ++j) acc[j] = Z[j * m + r];
                T a[PB];
#pragma unroll
                for (int u = 0; u < PB; ++u) a[u] = u < nb ? Lg[(size_t)(p0 + u) * m + r] : Sc<T>::zero();
#pragma unroll
                for (int u = 0; u < PB; ++u)
#pragma unroll
                    for (int j = 0; j < NS; ++j) fms_acc(acc[j], a[u], Z[j * m + p0 + u]);
#pragma unroll
                for (int j = 0; j < NS; ++j) Z[j * m + r] = acc[j];
            }
            __syncthreads();
        }
        // backward: L^T x = y, by panels from the last
        for (int p0 = (m - 1) / PB * PB; p0 >= 0; p0 -= PB) {
            const int nb = min(PB, m - p0);
            {   // y[p0 + t] -= sum over solved rows r >= p0 + nb of L(r, p0 + t) x_r: 16 threads per column t
                const int t = tid >> 4, sl = tid & 15;
                T part[NS];
#pragma unroll
                for (int j = 0; j < NS; ++j) part[j] = Sc<T>::zero();
                if (t < nb) {
                    const T* col = Lg + (size_t)(p0 + t) * m;
#pragma unroll 4
                    for (int r = p0 + nb + sl; r < m; r += 16) {
                        const T a = col[r];
#pragma unroll
                        for (int j = 0; j < NS; ++j) fma_acc(part[j], a, Z[j * m + r]);
                    }
                }
#pragma unroll
                for (int j = 0; j < NS; ++j) {
#pragma unroll
                    for (int off = 8; off > 0; off >>= 1) part[j] += shfl_xor_t(part[j], off);
                }
                __syncthreads();
                if (sl == 0 && t < nb)
#pragma unroll
                    for (int j = 0; j < NS; ++j) Z[j * m + p0 + t] -= part[j];
            }
            stage_diag(p0, nb);
            __syncthreads();
            if (warp < NS) {   // the panel's triangle of L^T, lane t = row p0 + t
                const int j = warp;
                T v = lane < nb ? Z[j * m + p0 + lane] : Sc<T>::zero();
#pragma unroll
                for (int u = PB - 1; u >= 0; --u) {
                    if (u < nb) {
                        if (lane == u) v = Sc<T>::mul(v, Sc<T>::recip(Ld[u][u]));
                        const T xu = shfl_w(v, u, 32);
                        if (lane < u) fms_acc(v, Ld[lane][u], xu);
                    }
                }
                if (lane < nb) Z[j * m + p0 + lane] = v;
            }
            __syncthreads();
        }
        // x += z; convergence: max |z| <= tol max |x| per system
        if (tid < NS) {
            s_dx[tid] = 0.0;
            s_x[tid] = 0.0;
        }
        __syncthreads();
        {
            // the NT / NS threads of system j (NT / NS a multiple of 32):
            // rows r = i, i + NT / NS, ..., then their warps
            constexpr int TPS = NT / NS;
            static_assert(TPS % 32 == 0, "whole warps per system");
            const int j = tid / TPS, i = tid % TPS;
            double dmax = 0.0, xmax = 0.0;
            for (int r = i; r < m; r += TPS) {
                const T z = Z[j * m + r];
                const T x = X[j * m + r] + z;
                X[j * m + r] = x;
                dmax = fmax(dmax, mag1(z));
                xmax = fmax(xmax, mag1(x));
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
                xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, off));
            }
            if (lane == 0) {
                atomicMax(reinterpret_cast<unsigned long long*>(&s_dx[j]), __double_as_longlong(dmax));
                atomicMax(reinterpret_cast<unsigned long long*>(&s_x[j]), __double_as_longlong(xmax));
            }
        }
        __syncthreads();
        if (tid == 0) {
            // converged: the correction at tol of the solution, or no longer
            // contracting at the rounding level of the residual (a small
            // correction that did not halve)
            int go = 0;
            for (int j = 0; j < ns; ++j) {
                const bool done = s_dx[j] <= tol * s_x[j] ||
                                  (it >= 2 && s_dx[j] > 0.5 * s_dprev[j] && s_dx[j] <= 1e-9 * s_x[j]);
                go |= !done;
                s_dprev[j] = s_dx[j];
            }
            s_go = go;
        }
        __syncthreads();
        if (!s_go) break;
        if (it + 1 >= maxit) {
            if (tid == 0) atomicAdd(nonconv, ns);
            return;
        }
    }
    if (tid == 0) atomicAdd(nonconv + 1, ns * (it + 1));   // system-iterations, for the work count
    for (int i = tid; i < m * ns; i += NT) {
        const int j = i / m, r = i % m;
        xg[((size_t)k * L + l0 + j) * m + r] = X[j * m + r];
    }
}

// ---------------------------------------------------------------------------
// z^_l = u^_l - V^ p_G: tiles of 64 interior rows x 32 electrodes; the
// boundary columns in the order of their first row, so a tile stops at the
// first column that is zero on all its rows.
template <typename T>
__global__ void __launch_bounds__(128) k_schur_zrebuild(SchurArgs s, T* X, const T* __restrict__ xg)
{
    constexpr int TI = 64, TL = 32, TG = 16;
    extern __shared__ __align__(16) unsigned char zr_dyn[];   // both stages of both tiles
    auto As = reinterpret_cast<T(*)[TG][TI + 1]>(zr_dyn);                                  // [2][TG][TI + 1]
    auto Bs = reinterpret_cast<T(*)[TG][TL + 1]>(zr_dyn + 2 * TG * (TI + 1) * sizeof(T));  // [2][TG][TL + 1]
    const int tid = threadIdx.x;
    // wavenumbers along x and the row blocks from the last: a late row block
    // meets the most boundary columns, so the longest tiles start first
    const int k = s.k0 + blockIdx.x, i0 = (gridDim.y - 1 - blockIdx.y) * TI, l0 = blockIdx.z * TL;
    const int ti = tid % 16, tl = tid / 16;
    const int m = s.m, nI = s.nI, L = s.L;
    T* Xk = X + (size_t)k * s.ncol * nI;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = Sc<T>::zero();
    // boundary columns [q0, q0 + TG) of both operands into buffer `buf`
    // (cp.async, the next block's copies in flight during this one)
    auto stage = [&](int buf, int q0) {
        for (int idx = tid; idx < TG * TI; idx += 128) {
            const int gg = idx / TI, ii = idx % TI;
            const int g = q0 + gg < m ? s.gsort[q0 + gg] : -1;
            if (g >= 0 && i0 + ii < nI) cp_async_elem<T>(&As[buf][gg][ii], Xk + (size_t)(L + g) * nI + i0 + ii);
            else As[buf][gg][ii] = Sc<T>::zero();
        }
        for (int idx = tid; idx < TG * TL; idx += 128) {
            const int ll = idx / TG, gg = idx % TG;
            const int g = q0 + gg < m ? s.gsort[q0 + gg] : -1;
            if (g >= 0 && l0 + ll < L) cp_async_elem<T>(&Bs[buf][gg][ll], xg + ((size_t)k * L + l0 + ll) * m + g);
            else Bs[buf][gg][ll] = Sc<T>::zero();
        }
        cp_async_commit();
    };
    // the boundary columns in the order of their first rows: a block whose
    // first column starts below this tile ends the loop
    auto live = [&](int q0) { return q0 < m && s.gfirst[q0] < i0 + TI; };
    int buf = 0;
    if (live(0)) stage(0, 0);
    for (int q0 = 0; live(q0); q0 += TG, buf ^= 1) {
        if (live(q0 + TG)) {
            stage(buf ^ 1, q0 + TG);   // its last readers finished before the trailing barrier
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();
#pragma unroll 4
        for (int gg = 0; gg < TG; ++gg) {
            T a4[4], b4[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) a4[a] = As[buf][gg][ti + 16 * a];
#pragma unroll
            for (int c = 0; c < 4; ++c) b4[c] = Bs[buf][gg][tl + 8 * c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) fma_acc(acc[a][c], a4[a], b4[c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int l = l0 + tl + 8 * c;
        if (l >= L) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ti + 16 * a;
            if (i < nI) Xk[(size_t)l * nI + i] -= acc[a][c];
        }
    }
}

template <typename T>
__global__ void k_schur_out_gam(SchurArgs s, const T* __restrict__ xg, int n, cd* kpot)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.nk * s.L * s.m) return;
    const int g = (int)(idx % s.m);
    const long long kl = (long long)s.k0 * s.L + idx / s.m;   // k L + l
    kpot[kl * n + s.gam[g]] = Sc<T>::to_cd(xg[kl * s.m + g]);
}

// window rows: mb + 3 BB (the rows of a block, the band below it, and two
// blocks arriving ahead), a multiple of BB
int sweep_wz(int mbI) { return (mbI + 4 * SCHUR_MS_BB - 1) / SCHUR_MS_BB * SCHUR_MS_BB; }

constexpr int SWEEP_NT = 288;   // 4 x 4 update tiles of a 129-row band at R = 32 in one round

// Columns per update tile of the sweeps: 2 (twice the threads, each with
// half the accumulators) or 4.  Measured on the 60k-triangle mesh with the
// half-warp triangles: back sweep and rebuild 20.6 ms with 2 against 24.0
// with 4, the forward sweep's part after the factor 11.7 against 12.5;
// CRT_B200_SCHUR_TILE=4 selects the wider tiles.
static int sweep_tc(bool)
{
    const char* v = std::getenv("CRT_B200_SCHUR_TILE");
    return (v && std::strcmp(v, "4") == 0) ? 4 : 2;
}

}  // namespace

// ---------------------------------------------------------------------------
template <typename T>
size_t schur_sweep_smem(int mbI, int WI, int R)
{
    return (size_t)2 * SCHUR_MS_BB * WI * sizeof(T) + (size_t)sweep_wz(mbI) * R * sizeof(T);
}

template <typename T>
void launch_schur_rhs(const SchurArgs& s, const BandArgs<T>& full, const double* fakws, T* X, T* cval, cudaStream_t st)
{
    const int ns = s.K * s.L;
    k_schur_rhs_src<T><<<(ns + 127) / 128, 128, 0, st>>>(s, fakws, X);
    const long long nc = (long long)s.K * s.ncpl;
    if (nc > 0) k_schur_rhs_cpl<T><<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(s, full, fakws, X, cval);
}

template <typename T>
void launch_schur_transpose(const SchurArgs& s, const T* Lws, T* Lrev, cudaStream_t st)
{
    const long long tot = (long long)s.nk * s.nI * s.WI;
    k_schur_transpose<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, Lws, Lrev);
}

template <typename T>
void launch_schur_forward(const SchurArgs& s, const T* Lws, T* X, cudaStream_t st)
{
    const size_t smem = schur_sweep_smem<T>(s.mbI, s.WI, s.R);
    dim3 grid(s.nk, s.nblk);
    auto go = [&](auto kern, int nt) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, nt, smem, st>>>(s, Lws, nullptr, X, nullptr, 0, sweep_wz(s.mbI), 0, 2);
    };
    // update tiles of 4 rows x TC columns: one round of a 129-row band
    const bool narrow = sweep_tc(false) == 2;
    const size_t smem_pp = (size_t)3 * SCHUR_MS_BB * s.WI * sizeof(T) + (size_t)sweep_wz(s.mbI) * 16 * sizeof(T);
    const char* fv = std::getenv("CRT_B200_SCHUR_FWD");
    if (s.R == 16 && fv && std::strcmp(fv, "pp") == 0 && smem_pp <= 227 * 1024) {
        // 16-column blocks: the triangle beside the update (as the back sweep)
        cudaFuncSetAttribute(k_schur_sweep_pp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_pp);
        k_schur_sweep_pp<T><<<grid, 512, smem_pp, st>>>(s, Lws, nullptr, X, nullptr, 0, sweep_wz(s.mbI), 0);
        return;
    }
    // 16-column blocks, rows one block ahead: the window of mb + 2 BB rows
    // lets two CTAs share an SM (2 x 113 KB with the driver's reserve)
    const int wz1 = (s.mbI + 2 * SCHUR_MS_BB + SCHUR_MS_BB - 1) / SCHUR_MS_BB * SCHUR_MS_BB;
    const size_t smem1 = (size_t)2 * SCHUR_MS_BB * s.WI * sizeof(T) + (size_t)wz1 * 16 * sizeof(T);
    if (s.R == 16 && !(fv && std::strcmp(fv, "wide") == 0) && 2 * (smem1 + 2048) <= 228 * 1024) {
        auto kern = k_schur_sweep<T, 288, 16, SCHUR_MS_BB, 2, 2>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
        kern<<<grid, 288, smem1, st>>>(s, Lws, nullptr, X, nullptr, 0, wz1, 0, 1);
        return;
    }
    if (s.R == 16) {
        if (narrow) go(k_schur_sweep<T, 288, 16, SCHUR_MS_BB, 2>, 288);
        else go(k_schur_sweep<T, 160, 16, SCHUR_MS_BB, 4>, 160);
    } else {
        if (narrow) go(k_schur_sweep<T, 544, SCHUR_MS_R, SCHUR_MS_BB, 2>, 544);
        else go(k_schur_sweep<T, SWEEP_NT, SCHUR_MS_R, SCHUR_MS_BB, 4>, SWEEP_NT);
    }
}

// One thread: returns once `want` CTAs of the concurrent factor have begun
// (bounded: about 2 s), so that the sweep's CTAs, which wait on that
// factor's progress, never take SMs the factor still needs.
__global__ void k_wait_started(const int* started, int want, int* status)
{
    long polls = 0;
    while (*(volatile const int*)started < want) {
        if (++polls > (1L << 21)) {
            atomicMax(status, (int)CRT_ERR_CUDA);
            return;
        }
        __nanosleep(1000);
    }
}

void launch_wait_started(const int* started, int want, int* status, cudaStream_t st)
{
    k_wait_started<<<1, 1, 0, st>>>(started, want, status);
}

template <typename T>
void launch_schur_gram(const SchurArgs& s, const T* X, T* C, cudaStream_t st)
{
    dim3 grid(s.nk, (s.m + 63) / 64, (s.ncol + 31) / 32);
    const int smem = 2 * 16 * (64 + 1 + 32 + 1) * (int)sizeof(T);   // the two stages of both tiles
    cudaFuncSetAttribute(k_schur_gram<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_schur_gram<T><<<grid, 128, smem, st>>>(s, X, C);
}

template <typename T>
void launch_schur_chol(const SchurArgs& s, const BandArgs<T>& full, const T* C, T* Sws, T* xg, int sys0, int nsys,
                       cudaStream_t st)
{
    // one CTA per SM with 16-column panels and the register prefetch, or two
    // CTAs per SM with 12-column panels where two such panels fit
    // (CRT_B200_SCHUR_CHOL=1 / 2 forces the form)
    constexpr int NT = 256;
    const size_t smem16 = ((size_t)16 * s.m + s.m) * sizeof(T), smem12 = ((size_t)12 * s.m + s.m) * sizeof(T);
    const char* ev = std::getenv("CRT_B200_SCHUR_CHOL");
    bool two = 2 * (smem12 + 1024) <= 227 * 1024;
    if (ev && std::strcmp(ev, "1") == 0) two = false;
    if (ev && std::strcmp(ev, "2") == 0 && 2 * (smem12 + 1024) <= 227 * 1024) two = true;
    if (two) {
        auto kern = k_schur_chol<T, NT, 12, false>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem12);
        kern<<<nsys, NT, smem12, st>>>(s, full, C, Sws, xg, sys0, nullptr);
    } else {
        auto kern = k_schur_chol<T, NT, 16, true>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem16);
        kern<<<nsys, NT, smem16, st>>>(s, full, C, Sws, xg, sys0, nullptr);
    }
}

template <typename T>
void launch_schur_s0(const SchurArgs& s, const BandArgs<T>& full, const T* C, T* S0, cudaStream_t st)
{
    const long long tot = (long long)s.K * s.m * s.m;
    k_schur_s0_vv<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, C, S0);
    const long long ng = (long long)s.K * s.ngg;
    if (ng > 0) k_schur_s0_area<T><<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(s, full, S0);
}

template <typename T>
void launch_schur_ref(const SchurArgs& s, const BandArgs<T>& full, const T* S0, T* Lref, int* nonconv, cudaStream_t st)
{
    constexpr int NT = 256;
    const size_t smem12 = ((size_t)12 * s.m + s.m) * sizeof(T), smem16 = ((size_t)16 * s.m + s.m) * sizeof(T);
    const int nref = s.K * s.ngrp;
    if (2 * (smem12 + 1024) <= 227 * 1024) {
        auto kern = k_schur_chol<T, NT, 12, false, true>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem12);
        kern<<<nref, NT, smem12, st>>>(s, full, S0, Lref, nullptr, 0, nonconv);
    } else {
        auto kern = k_schur_chol<T, NT, 16, true, true>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem16);
        kern<<<nref, NT, smem16, st>>>(s, full, S0, Lref, nullptr, 0, nonconv);
    }
}

template <typename T>
size_t schur_iter_smem(int m) { return 2 * (size_t)m * SCHUR_IT_NS * sizeof(T); }

template <typename T>
void launch_schur_dvals(const SchurArgs& s, const BandArgs<T>& full, T* Dv, cudaStream_t st)
{
    const long long tot = (long long)s.K * s.L * s.nbd;
    if (tot > 0) k_schur_dvals<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, full, Dv);
}

template <typename T>
void launch_schur_iter(const SchurArgs& s, const BandArgs<T>& full, const T* C, const T* S0, const T* Lref,
                       const T* Dv, T* xg, int maxit, double tol, int* nonconv, cudaStream_t st)
{
    // four systems per CTA at two CTAs per SM (electrode solves 13.6 against
    // 15.9 ms with eight at one on the 60k-triangle mesh: the panel solves
    // are chains of dependent steps, and two CTAs hide each other's
    // latency; two systems at three CTAs per SM measured 14.8 ms);
    // CRT_B200_SCHUR_IT_NS=8 keeps eight
    const char* nv = std::getenv("CRT_B200_SCHUR_IT_NS");
    if (!(nv && std::strcmp(nv, "8") == 0) && 2 * (2 * (size_t)s.m * 4 * sizeof(T)) <= 227 * 1024) {
        const size_t smem = 2 * (size_t)s.m * 4 * sizeof(T);
        const int cpg = (s.grp + 3) / 4;
        auto kern = k_schur_iter<T, 4, 2>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<s.K * s.ngrp * cpg, SCHUR_IT_NT, smem, st>>>(s, full, C, S0, Lref, Dv, xg, maxit, tol, nonconv);
        return;
    }
    const size_t smem = schur_iter_smem<T>(s.m);
    const int cpg = (s.grp + SCHUR_IT_NS - 1) / SCHUR_IT_NS;
    auto kern = k_schur_iter<T>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<s.K * s.ngrp * cpg, SCHUR_IT_NT, smem, st>>>(s, full, C, S0, Lref, Dv, xg, maxit, tol, nonconv);
}

template <typename T>
void launch_schur_zrebuild(const SchurArgs& s, T* X, const T* xg, cudaStream_t st)
{
    dim3 grid(s.nk, (s.nI + 63) / 64, (s.L + 31) / 32);
    const int smem = 2 * 16 * (64 + 1 + 32 + 1) * (int)sizeof(T);   // the two stages of both tiles
    cudaFuncSetAttribute(k_schur_zrebuild<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_schur_zrebuild<T><<<grid, 128, smem, st>>>(s, X, xg);
}

template <typename T>
void launch_schur_back(const SchurArgs& s, const T* Lrev, const double* fakws, const T* X, const T* xg, int n,
                       cd* kpot, cudaStream_t st)
{
    dim3 grid(s.nk, (s.L + SCHUR_BK_R - 1) / SCHUR_BK_R);
    // the triangle beside the update (three factor buffers; 16.4 against
    // 20.5 ms for back sweep and rebuild on the 60k-triangle mesh), unless
    // CRT_B200_SCHUR_BACK_PP=0 or its buffers do not fit
    const char* pv = std::getenv("CRT_B200_SCHUR_BACK_PP");
    const size_t smem_pp = (size_t)3 * SCHUR_MS_BB * s.WI * sizeof(T) + (size_t)sweep_wz(s.mbI) * 16 * sizeof(T);
    if (!(pv && std::strcmp(pv, "0") == 0) && smem_pp <= 227 * 1024) {
        cudaFuncSetAttribute(k_schur_sweep_pp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_pp);
        k_schur_sweep_pp<T><<<grid, 512, smem_pp, st>>>(s, Lrev, fakws, const_cast<T*>(X), kpot, n, sweep_wz(s.mbI), 1);
        const long long tot = (long long)s.nk * s.L * s.m;
        k_schur_out_gam<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, xg, n, kpot);
        return;
    }
    const size_t smem = schur_sweep_smem<T>(s.mbI, s.WI, SCHUR_BK_R);
    auto go = [&](auto kern, int nt) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, nt, smem, st>>>(s, Lrev, fakws, const_cast<T*>(X), kpot, n, sweep_wz(s.mbI), 1, 2);
    };
    // 4 x 2 update tiles of a 129-row band at R = 16 in one round (288
    // threads), or 4 x 4 (160)
    if (sweep_tc(true) == 2) go(k_schur_sweep<T, 288, SCHUR_BK_R, SCHUR_MS_BB, 2>, 288);
    else go(k_schur_sweep<T, 160, SCHUR_BK_R, SCHUR_MS_BB, 4>, 160);
    const long long tot = (long long)s.nk * s.L * s.m;
    k_schur_out_gam<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, xg, n, kpot);
}

template size_t schur_sweep_smem<cd>(int, int, int);
template size_t schur_sweep_smem<double>(int, int, int);
template void launch_schur_rhs<cd>(const SchurArgs&, const BandArgs<cd>&, const double*, cd*, cd*, cudaStream_t);
template void launch_schur_rhs<double>(const SchurArgs&, const BandArgs<double>&, const double*, double*, double*,
                                       cudaStream_t);
template void launch_schur_transpose<cd>(const SchurArgs&, const cd*, cd*, cudaStream_t);
template void launch_schur_transpose<double>(const SchurArgs&, const double*, double*, cudaStream_t);
template void launch_schur_forward<cd>(const SchurArgs&, const cd*, cd*, cudaStream_t);
template void launch_schur_forward<double>(const SchurArgs&, const double*, double*, cudaStream_t);
template void launch_schur_gram<cd>(const SchurArgs&, const cd*, cd*, cudaStream_t);
template void launch_schur_gram<double>(const SchurArgs&, const double*, double*, cudaStream_t);
template void launch_schur_chol<cd>(const SchurArgs&, const BandArgs<cd>&, const cd*, cd*, cd*, int, int, cudaStream_t);
template void launch_schur_chol<double>(const SchurArgs&, const BandArgs<double>&, const double*, double*, double*,
                                        int, int, cudaStream_t);
template void launch_schur_zrebuild<cd>(const SchurArgs&, cd*, const cd*, cudaStream_t);
template void launch_schur_zrebuild<double>(const SchurArgs&, double*, const double*, cudaStream_t);
template void launch_schur_back<cd>(const SchurArgs&, const cd*, const double*, const cd*, const cd*, int, cd*,
                                    cudaStream_t);
template void launch_schur_back<double>(const SchurArgs&, const double*, const double*, const double*, const double*,
                                        int, cd*, cudaStream_t);
template void launch_schur_s0<cd>(const SchurArgs&, const BandArgs<cd>&, const cd*, cd*, cudaStream_t);
template void launch_schur_s0<double>(const SchurArgs&, const BandArgs<double>&, const double*, double*, cudaStream_t);
template void launch_schur_ref<cd>(const SchurArgs&, const BandArgs<cd>&, const cd*, cd*, int*, cudaStream_t);
template void launch_schur_ref<double>(const SchurArgs&, const BandArgs<double>&, const double*, double*, int*,
                                       cudaStream_t);
template void launch_schur_dvals<cd>(const SchurArgs&, const BandArgs<cd>&, cd*, cudaStream_t);
template void launch_schur_dvals<double>(const SchurArgs&, const BandArgs<double>&, double*, cudaStream_t);
template void launch_schur_iter<cd>(const SchurArgs&, const BandArgs<cd>&, const cd*, const cd*, const cd*,
                                    const cd*, cd*, int, double, int*, cudaStream_t);
template void launch_schur_iter<double>(const SchurArgs&, const BandArgs<double>&, const double*, const double*,
                                        const double*, const double*, double*, int, double, int*, cudaStream_t);
template size_t schur_iter_smem<cd>(int);
template size_t schur_iter_smem<double>(int);
