// crt_schur.cu -- forward model by elimination of the mixed-boundary nodes
// (see crt_schur.h for the algebra).  Kernels:
//
//   k_schur_rhs_src / k_schur_rhs_cpl  right-hand sides [r_I | A_IG] of the
//       multi-RHS solve, one column per source electrode and per boundary
//       node, and the coupling values a(g, i) kept for the later steps;
//   k_schur_msolve  forward and back substitution of SCHUR_MS_R columns per
//       CTA against one wavenumber's interior factor: the factor streams
//       through shared memory in blocks of SCHUR_MS_BB columns (one bulk
//       copy per block, double-buffered, bounded mbarrier wait), the
//       right-hand sides live in a sliding window of rows; each block is a
//       16-row triangle (one half-warp per column, shuffle broadcasts) and a
//       (mb x 16) x (16 x 32) update of the rows below it (4 x 4 register
//       tiles) -- in the back pass the mirrored dot products;
//   k_schur_s0      S0 = -A_GI Y per wavenumber;
//   k_schur_chol    per (k, l): S_l = S0 + A_GG(l), right-looking blocked
//       Cholesky (unconjugated, complex symmetric as src/chol.f90:44-78)
//       with a 16-column panel in shared memory and 4 x 4 register tiles for
//       the trailing update, then the two triangular solves for p_G;
//   k_schur_out     kpot = w - Y p_G (a 64 x 32 tiled GEMM per wavenumber)
//       on the interior rows, p_G on the boundary rows.
#include "crt_schur.h"

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <utility>

// ---------------------------------------------------------------------------
// Host plan.
int schur_plan_host(const AssemblyLists& full, int n, const std::vector<int>& gamma_nodes,
                    const std::vector<int>& enr0, int lsink, int nsink0, SchurHost& o)
{
    o = SchurHost{};
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
    // columns by their first non-zero row, so that a block's forward pass
    // starts where its earliest column does
    const int ncol = o.L + o.m;
    o.col_order.resize(ncol);
    std::iota(o.col_order.begin(), o.col_order.end(), 0);
    std::stable_sort(o.col_order.begin(), o.col_order.end(), [&](int a, int b) { return first[a] < first[b]; });
    for (int b0 = 0; b0 < ncol; b0 += SCHUR_MS_R) {
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
template <typename T> __device__ __forceinline__ T shfl_xor1(T v);
template <> __device__ __forceinline__ double shfl_xor1<double>(double v) { return __shfl_xor_sync(0xffffffffu, v, 1); }
template <> __device__ __forceinline__ cd shfl_xor1<cd>(cd v)
{
    return cd{__shfl_xor_sync(0xffffffffu, v.x, 1), __shfl_xor_sync(0xffffffffu, v.y, 1)};
}
template <typename T> __device__ __forceinline__ T shfl_down_full(T v, int off);
template <> __device__ __forceinline__ double shfl_down_full<double>(double v, int off)
{
    return __shfl_down_sync(0xffffffffu, v, off);
}
template <> __device__ __forceinline__ cd shfl_down_full<cd>(cd v, int off)
{
    return cd{__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off)};
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

// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_schur_rhs_src(SchurArgs s, T* X)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= s.K * s.L) return;
    const int k = idx / s.L, l = idx % s.L;
    T* col = X + ((size_t)k * s.ncol + l) * s.nI;
    // r = e_src - e_sink (A pot = r; the reference's b = -r, src/kompab.f90)
    if (s.posI_src[l] >= 0) col[s.posI_src[l]] = Sc<T>::one();
    if (s.lsink && s.posI_sink >= 0) col[s.posI_sink] -= Sc<T>::one();
}

template <typename T>
__global__ void k_schur_rhs_cpl(SchurArgs s, BandArgs<T> A, T* X, T* cval)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.K * s.ncpl) return;
    const int k = (int)(idx / s.ncpl), q = (int)(idx % s.ncpl);
    // an interior-boundary entry has area contributions only (l unused)
    const T a = band_assemble_entry<T>(A, s.gi_ent[q], k, 0);
    cval[idx] = a;
    X[((size_t)k * s.ncol + s.L + s.gi_g[q]) * s.nI + s.gi_pos[q]] = a;
}

// ---------------------------------------------------------------------------
// Multi-RHS band solve: grid (column blocks, K).  Window Z[WZ][R] in shared
// memory, row r at slot r mod WZ, WZ >= mb + 2 BB so that the rows entering
// for the next block never share a slot with a row still in use.
template <typename T, int NT, int R, int BB>
__global__ void __launch_bounds__(NT, 1) k_schur_msolve(SchurArgs s, const T* __restrict__ Lws, size_t lstride,
                                                        const double* __restrict__ fakws, T* X, int WZ)
{
    static_assert(BB == 16 && R % 4 == 0 && NT % 16 == 0 && R % (NT / 16) == 0, "msolve layout");
    extern __shared__ __align__(16) unsigned char ms_dyn[];
    const int W = s.WI, n = s.nI, mb = s.mbI;
    T* Lb = reinterpret_cast<T*>(ms_dyn);                              // [2][BB * W]
    T* Z = Lb + 2 * BB * W;                                            // [WZ][R]
    double* fz = reinterpret_cast<double*>(Z + (size_t)WZ * R);        // [WZ]
    __shared__ T dinv[BB];
    __shared__ int colid[R];
    __shared__ __align__(8) unsigned long long bar[2];
    __shared__ int s_err;
    const int tid = threadIdx.x;
    const int blk = blockIdx.x, k = blockIdx.y;
    const int start = s.blk_start[blk];
    if (start >= n) return;   // every column of the block is zero, and so is its solution
    const T* Lk = Lws + (size_t)k * lstride;
    const double* fk = fakws + (size_t)k * n;
    if (tid < R) {
        const int c = blk * R + tid;
        colid[tid] = c < s.ncol ? s.col_order[c] : -1;
    }
    if (tid == 0) {
        s_err = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    __syncthreads();
    int ph[2] = {0, 0};
    auto colp = [&](int j) { return X + ((size_t)k * s.ncol + colid[j]) * n; };
    // factor columns [c0, c0 + nb) (one contiguous run of the column-packed
    // factor) into buffer `buf` by one bulk copy
    auto fetch = [&](int c0, int buf) {
        if (tid == 0) {
            const int nb = min(BB, n - c0);
            const int bytes = nb * W * (int)sizeof(T);
            mbar_expect_tx(&bar[buf], bytes);
            bulk_g2s(Lb + (size_t)buf * BB * W, Lk + (size_t)c0 * W, bytes, &bar[buf]);
        }
    };
    auto wait = [&](int buf) {
        if (!mbar_wait(&bar[buf], ph[buf])) s_err = 1;
        ph[buf] ^= 1;
    };
    // rows [r0, r1) of every column into the window; scaled (fak o b) for
    // the forward pass, as stored (z) for the back pass
    auto load_rows = [&](int r0, int r1, bool scale_in) {
        const int nr = r1 - r0;
        for (int idx = tid; idx < nr * R; idx += NT) {
            const int j = idx / nr, r = r0 + idx % nr;
            const double f = fk[r];
            T v = Sc<T>::zero();
            if (colid[j] >= 0) {
                v = colp(j)[r];
                if (scale_in) v = scale(v, f);
            }
            Z[(r % WZ) * R + j] = v;
            if (j == 0) fz[r % WZ] = f;
        }
    };

    // ---- forward substitution L z = fak o b from the block's first row
    load_rows(start, min(n, start + BB + mb), true);
    fetch(start, 0);
    int buf = 0;
    __syncthreads();
    for (int c0 = start; c0 < n; c0 += BB) {
        const int nb = min(BB, n - c0);
        wait(buf);
        if (c0 + BB < n) fetch(c0 + BB, buf ^ 1);
        const T* Lc = Lb + (size_t)buf * BB * W;
        if (tid < nb) dinv[tid] = Sc<T>::recip(Lc[tid * W]);
        __syncthreads();
        {   // the block's triangle: one half-warp per column, lane t = row c0 + t
            const int hw = tid >> 4, t = tid & 15;
            for (int j = hw; j < R; j += NT / 16) {
                T v = t < nb ? Z[((c0 + t) % WZ) * R + j] : Sc<T>::zero();
                for (int u = 0; u < nb; ++u) {
                    if (t == u) v = Sc<T>::mul(v, dinv[u]);
                    const T y = shfl_w(v, u, 16);
                    if (t > u && t < nb && t - u <= mb) fms_acc(v, Lc[u * W + (t - u)], y);
                }
                if (t < nb) Z[((c0 + t) % WZ) * R + j] = v;
            }
        }
        __syncthreads();
        // the block's rows are final: out to X
        for (int idx = tid; idx < nb * R; idx += NT) {
            const int j = idx / nb, t = idx % nb;
            if (colid[j] >= 0) colp(j)[c0 + t] = Z[((c0 + t) % WZ) * R + j];
        }
        {   // rows [c0 + nb, c0 + nb + mb) take the block's columns
            const int rlo = c0 + nb, rhi = min(n, c0 + nb + mb);
            const int nq = (rhi - rlo + 3) / 4;
            for (int tile = tid; tile < nq * (R / 4); tile += NT) {
                const int r0 = rlo + 4 * (tile / (R / 4)), j0 = 4 * (tile % (R / 4));
                T acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        acc[a][c] = r0 + a < rhi ? Z[((r0 + a) % WZ) * R + j0 + c] : Sc<T>::zero();
                for (int u = 0; u < nb; ++u) {
                    T zc[4], lv[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) zc[c] = Z[((c0 + u) % WZ) * R + j0 + c];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int d = r0 + a - (c0 + u);
                        lv[a] = (r0 + a < rhi && d <= mb) ? Lc[u * W + d] : Sc<T>::zero();
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < 4; ++c) fms_acc(acc[a][c], lv[a], zc[c]);
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    if (r0 + a < rhi)
#pragma unroll
                        for (int c = 0; c < 4; ++c) Z[((r0 + a) % WZ) * R + j0 + c] = acc[a][c];
            }
        }
        // the rows the next block reaches enter the window
        if (c0 + BB < n) load_rows(min(n, c0 + BB + mb), min(n, c0 + 2 * BB + mb), true);
        // the buffer just read is the destination of the bulk copy after next
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        buf ^= 1;
    }

    // ---- back substitution L^T x = z from the last block; the window holds
    // the solved rows [c1, c1 + mb) and the block's z rows [c0, c1)
    const int last0 = (n - 1) / BB * BB;
    load_rows(last0, n, false);
    fetch(last0, buf);
    __syncthreads();
    for (int c0 = last0; c0 >= 0; c0 -= BB) {
        const int nb = min(BB, n - c0), c1 = c0 + nb;
        wait(buf);
        if (c0 > 0) fetch(c0 - BB, buf ^ 1);
        const T* Lc = Lb + (size_t)buf * BB * W;
        if (tid < nb) dinv[tid] = Sc<T>::recip(Lc[tid * W]);
        {   // z_t -= sum over solved rows r >= c1 of L(r, c0 + t) x_r: thread
            // (t, 4 columns, half of the rows), halves combined by a shuffle
            const int half = tid & 1, combo = tid >> 1;
            const int t = combo >> 3, j0 = 4 * (combo & 7);
            T acc[4] = {Sc<T>::zero(), Sc<T>::zero(), Sc<T>::zero(), Sc<T>::zero()};
            if (t < nb) {
                const int rend = min(n, c0 + t + mb + 1);
                for (int r = c1 + half; r < rend; r += 2) {
                    const T lv = Lc[t * W + (r - c0 - t)];
#pragma unroll
                    for (int c = 0; c < 4; ++c) fma_acc(acc[c], lv, Z[(r % WZ) * R + j0 + c]);
                }
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[c] += shfl_xor1(acc[c]);
            if (half == 0 && t < nb)
#pragma unroll
                for (int c = 0; c < 4; ++c) Z[((c0 + t) % WZ) * R + j0 + c] -= acc[c];
        }
        __syncthreads();
        {   // the block's triangle of L^T, from its last row up
            const int hw = tid >> 4, t = tid & 15;
            for (int j = hw; j < R; j += NT / 16) {
                T v = t < nb ? Z[((c0 + t) % WZ) * R + j] : Sc<T>::zero();
                for (int u = nb - 1; u >= 0; --u) {
                    if (t == u) v = Sc<T>::mul(v, dinv[u]);
                    const T x = shfl_w(v, u, 16);
                    if (t < u && u - t <= mb) fms_acc(v, Lc[t * W + (u - t)], x);
                }
                if (t < nb) Z[((c0 + t) % WZ) * R + j] = v;
            }
        }
        __syncthreads();
        // x = fak o x^ out to X; the next block's z rows enter
        for (int idx = tid; idx < nb * R; idx += NT) {
            const int j = idx / nb, t = idx % nb;
            const int sl = (c0 + t) % WZ;
            if (colid[j] >= 0) colp(j)[c0 + t] = scale(Z[sl * R + j], fz[sl]);
        }
        if (c0 > 0) load_rows(c0 - BB, c0, false);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        buf ^= 1;
    }
    if (tid == 0 && s_err) atomicMax(&s.status[k], (int)CRT_ERR_CUDA);
}

// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_schur_s0(SchurArgs s, const T* __restrict__ X, const T* __restrict__ cval, T* S0)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long mm = (long long)s.m * s.m;
    if (idx >= (long long)s.K * mm) return;
    const int k = (int)(idx / mm);
    const int h = (int)((idx % mm) / s.m), g = (int)(idx % s.m);
    if (g < h) return;
    const T* Y = X + ((size_t)k * s.ncol + s.L + h) * s.nI;
    const T* cv = cval + (size_t)k * s.ncpl;
    T acc = Sc<T>::zero();
    for (int q = s.gi_ptr[g]; q < s.gi_ptr[g + 1]; ++q) fma_acc(acc, cv[q], Y[s.gi_pos[q]]);
    S0[(size_t)k * mm + (size_t)h * s.m + g] = -acc;
}

// ---------------------------------------------------------------------------
// Dense Cholesky of the Schur complements: one CTA per (k, l) system.
template <typename T, int NT, int NB>
__global__ void __launch_bounds__(NT, 1) k_schur_chol(SchurArgs s, BandArgs<T> A, const T* __restrict__ S0,
                                                      const T* __restrict__ X, const T* __restrict__ cval, T* Sws,
                                                      T* xg, int sys0)
{
    extern __shared__ __align__(16) unsigned char ch_dyn[];
    const int m = s.m;
    T* P = reinterpret_cast<T*>(ch_dyn);   // panel [NB][m]
    T* y = P + (size_t)NB * m;             // [m]
    __shared__ T red[NT / 32];
    __shared__ int s_err;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x, sys = sys0 + b, k = sys / s.L, l = sys % s.L;
    T* S = Sws + (size_t)b * m * m;
    const T* S0k = S0 + (size_t)k * m * m;
    if (tid == 0) s_err = 0;
    // S = S0[k] (lower triangle), plus A_GG(l)
    for (int c = 0; c < m; ++c)
        for (int r = c + tid; r < m; r += NT) S[(size_t)c * m + r] = S0k[(size_t)c * m + r];
    __syncthreads();
    for (int q = tid; q < s.ngg; q += NT) {
        const T a = band_assemble_entry<T>(A, s.gg_ent[q], k, l);
        S[(size_t)s.gg_h[q] * m + s.gg_g[q]] += a;
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
            __syncthreads();   // every thread has read the pivot
            for (int r = c + 1 + tid; r < m; r += NT) P[t * m + r] = Sc<T>::mul(P[t * m + r], inv);
            if (tid == 0) P[t * m + c] = root;
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
        // trailing update of the lower triangle below the panel, 4 x 4 tiles
        const int q0 = p0 + nb, mt = m - q0;
        if (mt > 0) {
            const int T4 = (mt + 3) / 4, ntile = T4 * (T4 + 1) / 2;
            for (int tile = tid; tile < ntile; tile += NT) {
                int X4 = (int)((sqrtf(8.0f * tile + 1.0f) - 1.0f) * 0.5f);
                while ((X4 + 1) * (X4 + 2) / 2 <= tile) ++X4;
                while (X4 * (X4 + 1) / 2 > tile) --X4;
                const int Y4 = tile - X4 * (X4 + 1) / 2;
                const int r0 = q0 + 4 * X4, cc0 = q0 + 4 * Y4;
                T acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int r = r0 + a, cc = cc0 + c;
                        acc[a][c] = (r < m && cc < m && r >= cc) ? S[(size_t)cc * m + r] : Sc<T>::zero();
                    }
                for (int t = 0; t < nb; ++t) {
                    T pr[4], pc[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        pr[a] = r0 + a < m ? P[t * m + r0 + a] : Sc<T>::zero();
                        pc[a] = cc0 + a < m ? P[t * m + cc0 + a] : Sc<T>::zero();
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < 4; ++c) fms_acc(acc[a][c], pr[a], pc[c]);
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int r = r0 + a, cc = cc0 + c;
                        if (r < m && cc < m && r >= cc) S[(size_t)cc * m + r] = acc[a][c];
                    }
            }
        }
        __syncthreads();
    }
    if (s_err) {
        if (tid == 0) atomicMax(&s.status[sys], s_err);
        return;
    }
    // right-hand side r_G - A_GI w_l
    const T* w = X + ((size_t)k * s.ncol + l) * s.nI;
    const T* cv = cval + (size_t)k * s.ncpl;
    for (int g = tid; g < m; g += NT) {
        T v = Sc<T>::zero();
        if (g == s.posG_src[l]) v = Sc<T>::one();
        if (s.lsink && g == s.posG_sink) v -= Sc<T>::one();
        for (int q = s.gi_ptr[g]; q < s.gi_ptr[g + 1]; ++q) fms_acc(v, cv[q], w[s.gi_pos[q]]);
        y[g] = v;
    }
    __syncthreads();
    // L y' = y, column by column
    for (int c = 0; c < m; ++c) {
        const T yc = Sc<T>::mul(y[c], Sc<T>::recip(S[(size_t)c * m + c]));
        __syncthreads();
        if (tid == 0) y[c] = yc;
        for (int r = c + 1 + tid; r < m; r += NT) fms_acc(y[r], S[(size_t)c * m + r], yc);
        __syncthreads();
    }
    // L^T x = y', one dot product per unknown from the last
    for (int c = m - 1; c >= 0; --c) {
        T part = Sc<T>::zero();
        for (int r = c + 1 + tid; r < m; r += NT) fma_acc(part, S[(size_t)c * m + r], y[r]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) part += shfl_down_full(part, off);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            T tot = Sc<T>::zero();
            for (int q = 0; q < NT / 32; ++q) tot += red[q];
            y[c] = Sc<T>::mul(y[c] - tot, Sc<T>::recip(S[(size_t)c * m + c]));
        }
        __syncthreads();
    }
    for (int g = tid; g < m; g += NT) xg[(size_t)sys * m + g] = y[g];
}

// ---------------------------------------------------------------------------
// kpot on the interior rows: w_l - Y p_G, tile 64 rows x 32 electrodes.
template <typename T>
__global__ void __launch_bounds__(128) k_schur_out(SchurArgs s, const T* __restrict__ X, const T* __restrict__ xg,
                                                   int n, cd* kpot)
{
    constexpr int TI = 64, TL = 32, TG = 16;
    __shared__ T As[TG][TI + 1];
    __shared__ T Bs[TG][TL + 1];
    const int tid = threadIdx.x;
    const int k = blockIdx.z, i0 = blockIdx.x * TI, l0 = blockIdx.y * TL;
    const int ti = tid % 16, tl = tid / 16;
    const int m = s.m, nI = s.nI;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = Sc<T>::zero();
    for (int g0 = 0; g0 < m; g0 += TG) {
        for (int idx = tid; idx < TG * TI; idx += 128) {
            const int gg = idx / TI, ii = idx % TI;
            As[gg][ii] = (g0 + gg < m && i0 + ii < nI) ? X[((size_t)k * s.ncol + s.L + g0 + gg) * nI + i0 + ii]
                                                       : Sc<T>::zero();
        }
        for (int idx = tid; idx < TG * TL; idx += 128) {
            const int ll = idx / TG, gg = idx % TG;
            Bs[gg][ll] = (g0 + gg < m && l0 + ll < s.L) ? xg[((size_t)k * s.L + l0 + ll) * m + g0 + gg] : Sc<T>::zero();
        }
        __syncthreads();
#pragma unroll 4
        for (int gg = 0; gg < TG; ++gg) {
            T a4[4], b4[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) a4[a] = As[gg][ti * 4 + a];
#pragma unroll
            for (int c = 0; c < 4; ++c) b4[c] = Bs[gg][tl * 4 + c];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) fma_acc(acc[a][c], a4[a], b4[c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int l = l0 + tl * 4 + c;
        if (l >= s.L) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ti * 4 + a;
            if (i >= nI) continue;
            const T v = X[((size_t)k * s.ncol + l) * nI + i] - acc[a][c];
            kpot[((size_t)k * s.L + l) * n + s.permI[i]] = Sc<T>::to_cd(v);
        }
    }
}

template <typename T>
__global__ void k_schur_out_gam(SchurArgs s, const T* __restrict__ xg, int n, cd* kpot)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)s.K * s.L * s.m) return;
    const int g = (int)(idx % s.m);
    const long long kl = idx / s.m;   // k L + l
    kpot[kl * n + s.gam[g]] = Sc<T>::to_cd(xg[idx]);
}

template <typename T>
int ms_wz(int mbI)
{
    return (mbI + 2 * SCHUR_MS_BB + SCHUR_MS_BB - 1) / SCHUR_MS_BB * SCHUR_MS_BB;
}

}  // namespace

// ---------------------------------------------------------------------------
template <typename T>
size_t schur_msolve_smem(int mbI, int WI)
{
    const int WZ = ms_wz<T>(mbI);
    return (size_t)2 * SCHUR_MS_BB * WI * sizeof(T) + (size_t)WZ * SCHUR_MS_R * sizeof(T) + (size_t)WZ * sizeof(double);
}

template <typename T>
void launch_schur_rhs(const SchurArgs& s, const BandArgs<T>& full, T* X, T* cval, cudaStream_t st)
{
    const int ns = s.K * s.L;
    k_schur_rhs_src<T><<<(ns + 127) / 128, 128, 0, st>>>(s, X);
    const long long nc = (long long)s.K * s.ncpl;
    if (nc > 0) k_schur_rhs_cpl<T><<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(s, full, X, cval);
}

template <typename T>
void launch_schur_msolve(const SchurArgs& s, const T* Lws, size_t lstride, const double* fakws, T* X, cudaStream_t st)
{
    constexpr int NT = 256;
    const size_t smem = schur_msolve_smem<T>(s.mbI, s.WI);
    auto kern = k_schur_msolve<T, NT, SCHUR_MS_R, SCHUR_MS_BB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(s.nblk, s.K);
    kern<<<grid, NT, smem, st>>>(s, Lws, lstride, fakws, X, ms_wz<T>(s.mbI));
}

template <typename T>
void launch_schur_s0(const SchurArgs& s, const T* X, const T* cval, T* S0, cudaStream_t st)
{
    const long long tot = (long long)s.K * s.m * s.m;
    k_schur_s0<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, X, cval, S0);
}

template <typename T>
void launch_schur_chol(const SchurArgs& s, const BandArgs<T>& full, const T* S0, const T* X, const T* cval, T* Sws,
                       T* xg, int sys0, int nsys, cudaStream_t st)
{
    constexpr int NT = 256, NB = 16;
    const size_t smem = ((size_t)NB * s.m + s.m) * sizeof(T);
    auto kern = k_schur_chol<T, NT, NB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<nsys, NT, smem, st>>>(s, full, S0, X, cval, Sws, xg, sys0);
}

template <typename T>
void launch_schur_out(const SchurArgs& s, const T* X, const T* xg, int n, cd* kpot, cudaStream_t st)
{
    dim3 grid((s.nI + 63) / 64, (s.L + 31) / 32, s.K);
    k_schur_out<T><<<grid, 128, 0, st>>>(s, X, xg, n, kpot);
    const long long tot = (long long)s.K * s.L * s.m;
    k_schur_out_gam<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, xg, n, kpot);
}

template size_t schur_msolve_smem<cd>(int, int);
template size_t schur_msolve_smem<double>(int, int);
template void launch_schur_rhs<cd>(const SchurArgs&, const BandArgs<cd>&, cd*, cd*, cudaStream_t);
template void launch_schur_rhs<double>(const SchurArgs&, const BandArgs<double>&, double*, double*, cudaStream_t);
template void launch_schur_msolve<cd>(const SchurArgs&, const cd*, size_t, const double*, cd*, cudaStream_t);
template void launch_schur_msolve<double>(const SchurArgs&, const double*, size_t, const double*, double*,
                                          cudaStream_t);
template void launch_schur_s0<cd>(const SchurArgs&, const cd*, const cd*, cd*, cudaStream_t);
template void launch_schur_s0<double>(const SchurArgs&, const double*, const double*, double*, cudaStream_t);
template void launch_schur_chol<cd>(const SchurArgs&, const BandArgs<cd>&, const cd*, const cd*, const cd*, cd*, cd*,
                                    int, int, cudaStream_t);
template void launch_schur_chol<double>(const SchurArgs&, const BandArgs<double>&, const double*, const double*,
                                        const double*, double*, double*, int, int, cudaStream_t);
template void launch_schur_out<cd>(const SchurArgs&, const cd*, const cd*, int, cd*, cudaStream_t);
template void launch_schur_out<double>(const SchurArgs&, const double*, const double*, int, cd*, cudaStream_t);
