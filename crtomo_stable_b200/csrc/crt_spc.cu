// crt_spc.cu -- block-tridiagonal preconditioner S^-1 for the normal-equation
// CG (the operator and its scaling are those of src/cg_mod.f90:426-726 and
// src/update.f90:200-231; the preconditioner itself has no counterpart in
// the reference, whose CG is preconditioned by cgfac alone).
//
// Host: reverse Cuthill-McKee (George-Liu pseudo-peripheral start, neighbours
// by ascending degree) on the graph of the roughness operator, block size
// B = roundup(bandwidth, 32), and one assembly entry per off-diagonal
// non-zero of R that lands in a diagonal block D_q or a sub-diagonal block
// F_q of the permuted matrix.
//
// Device, once per update:
//   k_spc_diag / k_spc_entries : S = I + lam C (R - diag R) C in blocks
//   k_spc_factor_v / k_spc_factor (one CTA) : T_q = D_q - F_q H_{q-1},
//                                H_{q-1} = T_{q-1}^-1 F_q^T, T_q^-1 by Gauss-Jordan
//                                with the block held in registers (SPD: no pivoting)
//   k_spc_gmul    (nb CTAs)    : G_q = T_q^-1 F_q
// and per CG iteration:
//   k_spc_u       (nb CTAs)    : u_q = T_q^-1 r_q on the permuted residual
//   k_spc_sweep   (one CTA)    : h_q = u_q - G_q h_{q-1}, x_q = h_q - H_q x_{q+1},
//                                z = x in element order (G and H column-major)
// The sub-diagonal blocks are stored transposed, FT_q[j][i] = F_q[i][j], so
// that both products of a block step read rows of their operands.
#include "crt_spc.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "crt_cg.h"

namespace {

constexpr int SPC_NT = 1024;

// ---------------------------------------------------------------------------
// host: ordering
//
// Per connected component: George-Liu pseudo-peripheral node r, then a
// Cuthill-McKee breadth-first numbering (neighbours by ascending degree,
// ties by index) from each of a few candidate roots -- r, the far end of
// its level structure and the lowest-degree nodes of the last level -- and
// the numbering with the smallest bandwidth is kept.  The concatenated
// order is reversed (which does not change the bandwidth).
void rcm_order(int M, const std::vector<int>& xadj, const std::vector<int>& adj, std::vector<int>& order)
{
    std::vector<int> deg(M), stamp(M, -1), lev(M, 0), queue, lpos(M, -1), cm, best;
    std::vector<char> placed(M, 0);
    for (int i = 0; i < M; ++i) deg[i] = xadj[i + 1] - xadj[i];
    queue.reserve(M);
    order.clear();
    order.reserve(M);
    int sid = 0;
    // BFS over the unplaced nodes reachable from root; returns the depth and
    // the lowest-degree node of the last level.
    auto bfs = [&](int root, int& depth, int& cand) {
        ++sid;
        queue.clear();
        queue.push_back(root);
        stamp[root] = sid;
        lev[root] = 0;
        for (size_t h = 0; h < queue.size(); ++h) {
            const int v = queue[h];
            for (int e = xadj[v]; e < xadj[v + 1]; ++e) {
                const int w = adj[e];
                if (placed[w] || stamp[w] == sid) continue;
                stamp[w] = sid;
                lev[w] = lev[v] + 1;
                queue.push_back(w);
            }
        }
        depth = lev[queue.back()];
        cand = queue.back();
        for (int v : queue)
            if (lev[v] == depth && deg[v] < deg[cand]) cand = v;
    };
    std::vector<int> nbr;
    // Cuthill-McKee numbering of the component from root into cm; returns
    // its bandwidth.
    auto cuthill_mckee = [&](int root) {
        ++sid;
        cm.clear();
        cm.push_back(root);
        stamp[root] = sid;
        for (size_t head = 0; head < cm.size(); ++head) {
            const int v = cm[head];
            nbr.clear();
            for (int e = xadj[v]; e < xadj[v + 1]; ++e)
                if (!placed[adj[e]] && stamp[adj[e]] != sid) nbr.push_back(adj[e]);
            std::sort(nbr.begin(), nbr.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            for (int w : nbr) {
                if (stamp[w] == sid) continue;
                stamp[w] = sid;
                cm.push_back(w);
            }
        }
        for (size_t k = 0; k < cm.size(); ++k) lpos[cm[k]] = (int)k;
        int bw = 0;
        for (int v : cm)
            for (int e = xadj[v]; e < xadj[v + 1]; ++e) bw = std::max(bw, std::abs(lpos[v] - lpos[adj[e]]));
        return bw;
    };
    for (int s0 = 0; s0 < M; ++s0) {
        if (placed[s0]) continue;
        int d0, x;
        bfs(s0, d0, x);
        int r = s0;
        for (int v : queue)
            if (deg[v] < deg[r]) r = v;
        bfs(r, d0, x);
        for (int it = 0; it < 16; ++it) {
            int dx, y;
            bfs(x, dx, y);
            if (dx <= d0) break;
            r = x;
            d0 = dx;
            x = y;
        }
        // candidate roots
        std::vector<int> cands{r, x};
        bfs(r, d0, x);
        std::vector<int> last;
        for (int v : queue)
            if (lev[v] == d0) last.push_back(v);
        std::sort(last.begin(), last.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
        for (size_t k = 0; k < last.size() && k < 4; ++k) cands.push_back(last[k]);
        int best_bw = -1;
        for (int c : cands) {
            const int bw = cuthill_mckee(c);
            if (best_bw < 0 || bw < best_bw) {
                best_bw = bw;
                best = cm;
            }
        }
        for (int v : best) {
            placed[v] = 1;
            order.push_back(v);
        }
    }
    std::reverse(order.begin(), order.end());
}

// ---------------------------------------------------------------------------
// device helpers
__device__ __forceinline__ float warp_allsum_f(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// f(integral_constant<int, i>) for i = 0 .. N-1, unrolled at compile time
template <typename F, int... I>
__device__ __forceinline__ void static_for_seq(F&& f, std::integer_sequence<int, I...>)
{
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
    static_for_seq(f, std::make_integer_sequence<int, N>{});
}

__global__ void k_spc_diag(float* DF, int nb, int B)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * B) return;
    const int q = idx / B, t = idx % B;
    DF[(size_t)q * B * B + (size_t)t * B + t] = 1.0f;
}

__global__ void k_spc_entries(const int4* __restrict__ ent, int nent, const double* __restrict__ cgfac,
                              const double* __restrict__ smatm, double lam, float* DF)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nent) return;
    const int4 e = ent[k];
    DF[e.x] = (float)(lam * cgfac[e.y] * smatm[e.w] * cgfac[e.z]);
}

// One CTA: the sequential block recurrence for B <= 128, with (B/8)^2
// threads; thread (ty, tx) owns an 8 x 8 set of a block's entries in
// registers: rows 8 ty .. 8 ty + 7 and the two column quads 4 tx .. 4 tx + 3
// and B/2 + 4 tx .. B/2 + 4 tx + 3 (so that the 16-byte loads of a quarter
// warp cover consecutive banks).  With X = T_{q-1}^-1 (symmetric) and FT_q
// in shared memory, both products take k-rows of their operands,
//   H[r][c] = sum_k X[k][r] FT[k][c],    T[r][c] = D[r][c] - sum_k FT[k][r] H[k][c],
// so each k step of a thread is four 16-byte shared loads and 64 FMAs; the
// Gauss-Jordan inversion publishes row and column k through double-buffered
// vectors (one barrier per step).  FT_{q+1} is copied into the other half of
// a shared double buffer by cp.async while block q is formed and inverted.
//
// With segs, CTA b runs the recurrence over the blocks segs[b].x ..
// segs[b].y only (a segment's interior, its first block without coupling);
// without, over 0 .. nb-1.  A non-positive pivot is reported through flag
// (zeroed by the caller).
template <int NB>
__global__ void __launch_bounds__(16 * NB * NB, 1) k_spc_factor_v(float* DF, float* H, int nb, int* flag,
                                                                   const int2* __restrict__ segs)
{
    constexpr int B = 32 * NB, TPR = B / 8, NT = TPR * TPR, HB = B / 2;
    extern __shared__ __align__(16) float smem[];
    float* X = smem;                  // [B][B]     T_{q-1}^-1, then H_{q-1}
    float* FTs = X + B * B;           // [2][B][B]  FT_q in half q & 1
    float* rowb = FTs + 2 * B * B;    // [2][B]
    float* colb = rowb + 2 * B;       // [2][B]
    const int tid = threadIdx.x, tx = tid % TPR, ty = tid / TPR;
    const int r0 = 8 * ty, c0 = 4 * tx;
    const size_t BB = (size_t)B * B;
    const float* F = DF + (size_t)nb * BB;
    auto cidx = [&](int b) { return (b >> 2) * HB + c0 + (b & 3); };
    auto stage_ft = [&](int q) {
        const float4* src = reinterpret_cast<const float4*>(F + (size_t)q * BB);
        float* dst = FTs + (size_t)(q & 1) * BB;
        for (int i = tid; i < (int)(BB / 4); i += NT) cp_async16(dst + 4 * i, src + i);
        cp_async_commit();
    };
    auto unpack = [](float4 a, float4 b, float (&v)[8]) {
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    };
    // 8 consecutive floats (rows) / this thread's two column quads of a row
    auto ld_rows = [&](const float* p, float (&v)[8]) {
        unpack(*reinterpret_cast<const float4*>(p), *reinterpret_cast<const float4*>(p + 4), v);
    };
    auto ld_cols = [&](const float* row, float (&v)[8]) {
        unpack(*reinterpret_cast<const float4*>(row + c0), *reinterpret_cast<const float4*>(row + HB + c0), v);
    };
    auto st_rows = [](float* p, const float (&v)[8]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<float4*>(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
    };
    auto st_cols = [&](float* row, const float (&v)[8]) {
        *reinterpret_cast<float4*>(row + c0) = make_float4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<float4*>(row + HB + c0) = make_float4(v[4], v[5], v[6], v[7]);
    };
    int first_bad = 0;
    const int2 sg = segs ? segs[blockIdx.x] : make_int2(0, nb - 1);
    const int qs = sg.x, qe = sg.y;
    if (qe > qs) stage_ft(qs + 1);
    for (int q = qs; q <= qe; ++q) {
        float* Dq = DF + (size_t)q * BB;
        float t[8][8];
#pragma unroll
        for (int a = 0; a < 8; ++a) ld_cols(Dq + (size_t)(r0 + a) * B, t[a]);
        if (q > qs) {
            if (q + 1 <= qe) {
                stage_ft(q + 1);            // the half of FT_{q-1}, long since read
                cp_async_wait_group<1>();   // FT_q has landed
            } else {
                cp_async_wait_all();
            }
            __syncthreads();
            const float* FT = FTs + (size_t)(q & 1) * BB;
            float h[8][8];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) h[a][b] = 0.0f;
#pragma unroll 2
            for (int k = 0; k < B; ++k) {
                float xa[8], fb[8];
                ld_rows(X + k * B + r0, xa);
                ld_cols(FT + k * B, fb);
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) h[a][b] = fmaf(xa[a], fb[b], h[a][b]);
            }
            __syncthreads();
#pragma unroll
            for (int a = 0; a < 8; ++a) st_cols(X + (r0 + a) * B, h[a]);
            // the sweep reads H_{q-1} column-major: HT[c][r] = H[r][c]
            float* Hq = H + (size_t)(q - 1) * BB;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                float col[8];
#pragma unroll
                for (int a = 0; a < 8; ++a) col[a] = h[a][b];
                st_rows(Hq + (size_t)cidx(b) * B + r0, col);
            }
            __syncthreads();
#pragma unroll 2
            for (int k = 0; k < B; ++k) {
                float fa[8], hb[8];
                ld_rows(FT + k * B + r0, fa);
                ld_cols(X + k * B, hb);
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) t[a][b] = fmaf(-fa[a], hb[b], t[a][b]);
            }
        }
        // Gauss-Jordan inversion in place (SPD, no pivoting).  Row k = 8 kq +
        // kr is held by the threads with ty = kq (entry kr); column k by those
        // with tx = (k mod B/2) / 4 (entry 4 (k >= B/2) + k % 4).  The eight
        // steps of a row group are unrolled, so a thread's entries of row and
        // column k are static register indices.
        auto gj_step = [&](const int k, auto kr_c, auto half_c) {
            constexpr int kr = decltype(kr_c)::value, kb = 4 * decltype(half_c)::value + (kr & 3);
            const int buf = (k & 1) * B;
            const bool row_own = ty == (k >> 3), col_own = tx == ((k % HB) >> 2);
            if (row_own) st_cols(rowb + buf, t[kr]);
            if (col_own) {
                float col[8];
#pragma unroll
                for (int a = 0; a < 8; ++a) col[a] = t[a][kb];
                st_rows(colb + buf + r0, col);
            }
            __syncthreads();
            float piv = rowb[buf + k];
            if (!(piv > 0.0f)) {
                if (first_bad == 0) first_bad = q + 1;
                piv = 1.0f;
            }
            const float pinv = __frcp_rn(piv);
            float cv[8], rv[8];
            ld_rows(colb + buf + r0, cv);
            ld_cols(rowb + buf, rv);
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const float ci = cv[a] * pinv;
#pragma unroll
                for (int b = 0; b < 8; ++b) t[a][b] = fmaf(-ci, rv[b], t[a][b]);
            }
            if (row_own) {
#pragma unroll
                for (int b = 0; b < 8; ++b) t[kr][b] = (cidx(b) == k) ? pinv : rv[b] * pinv;
            }
            if (col_own) {
#pragma unroll
                for (int a = 0; a < 8; ++a)
                    if (r0 + a != k) t[a][kb] = -cv[a] * pinv;
            }
        };
        for (int kq = 0; kq < TPR; ++kq) {
            if (kq < TPR / 2)
                static_for<8>([&](auto kr) { gj_step(8 * kq + decltype(kr)::value, kr, std::integral_constant<int, 0>{}); });
            else
                static_for<8>([&](auto kr) { gj_step(8 * kq + decltype(kr)::value, kr, std::integral_constant<int, 1>{}); });
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            st_cols(Dq + (size_t)(r0 + a) * B, t[a]);
            st_cols(X + (r0 + a) * B, t[a]);
        }
    }
    if (first_bad && tid == 0) atomicExch(flag, first_bad);
}

// One CTA: the sequential block recurrence, for B > 128 (every thread owns
// the NB x NB entries (ty + 32a, tx + 32b) of a block, operands staged in
// chunks of 32 k).
template <int NB>
__global__ void __launch_bounds__(SPC_NT, 1) k_spc_factor(float* DF, float* H, int nb, int* flag)
{
    constexpr int B = 32 * NB, LD = B + 1;
    extern __shared__ float smem[];
    float* X = smem;              // [B][LD]   T_{q-1}^-1, then H_{q-1}
    float* Sg = X + B * LD;       // [32][LD]  staged operand chunk
    float* rowb = Sg + 32 * LD;   // [2][B]
    float* colb = rowb + 2 * B;   // [2][B]
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const size_t BB = (size_t)B * B;
    const float* F = DF + (size_t)nb * BB;
    int first_bad = 0;
    for (int q = 0; q < nb; ++q) {
        float* Dq = DF + (size_t)q * BB;
        float t[NB][NB];
        if (q > 0) {
            const float* FTq = F + (size_t)q * BB;
            // H = T_{q-1}^-1 F_q^T:  H[r][c] = sum_k X[r][k] F_q[c][k]
            float h[NB][NB];
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) h[a][b] = 0.0f;
            for (int k0 = 0; k0 < B; k0 += 32) {
                __syncthreads();
                for (int u = tid; u < 32 * B; u += SPC_NT) {
                    const int c = u % B, kk = u / B;
                    Sg[kk * LD + c] = FTq[(size_t)(k0 + kk) * B + c];
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < 32; ++kk) {
                    float av[NB], bv[NB];
#pragma unroll
                    for (int a = 0; a < NB; ++a) av[a] = X[(ty + 32 * a) * LD + k0 + kk];
#pragma unroll
                    for (int b = 0; b < NB; ++b) bv[b] = Sg[kk * LD + tx + 32 * b];
#pragma unroll
                    for (int a = 0; a < NB; ++a)
#pragma unroll
                        for (int b = 0; b < NB; ++b) h[a][b] = fmaf(av[a], bv[b], h[a][b]);
                }
            }
            __syncthreads();
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) X[(ty + 32 * a) * LD + tx + 32 * b] = h[a][b];
            __syncthreads();
            // the sweep reads H_{q-1} column-major: HT[c][r] = H[r][c]
            float* Hq = H + (size_t)(q - 1) * BB;
            for (int u = tid; u < B * B; u += SPC_NT) {
                const int r = u % B, c = u / B;
                Hq[(size_t)c * B + r] = X[r * LD + c];
            }
            // T = D_q - F_q H
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) t[a][b] = Dq[(size_t)(ty + 32 * a) * B + tx + 32 * b];
            for (int k0 = 0; k0 < B; k0 += 32) {
                __syncthreads();
                for (int u = tid; u < 32 * B; u += SPC_NT) {
                    const int r = u % B, kk = u / B;
                    Sg[kk * LD + r] = FTq[(size_t)(k0 + kk) * B + r];
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < 32; ++kk) {
                    float av[NB], bv[NB];
#pragma unroll
                    for (int a = 0; a < NB; ++a) av[a] = Sg[kk * LD + ty + 32 * a];
#pragma unroll
                    for (int b = 0; b < NB; ++b) bv[b] = X[(k0 + kk) * LD + tx + 32 * b];
#pragma unroll
                    for (int a = 0; a < NB; ++a)
#pragma unroll
                        for (int b = 0; b < NB; ++b) t[a][b] = fmaf(-av[a], bv[b], t[a][b]);
                }
            }
        } else {
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) t[a][b] = Dq[(size_t)(ty + 32 * a) * B + tx + 32 * b];
        }
        // Gauss-Jordan inversion in place (SPD, no pivoting); row k and
        // column k are published through double-buffered shared vectors.
        for (int k = 0; k < B; ++k) {
            const int buf = (k & 1) * B, ka = k >> 5, kl = k & 31;
            if (ty == kl) {
#pragma unroll
                for (int a = 0; a < NB; ++a)
                    if (a == ka) {
#pragma unroll
                        for (int b = 0; b < NB; ++b) rowb[buf + tx + 32 * b] = t[a][b];
                    }
            }
            if (tx == kl) {
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    if (b == ka) {
#pragma unroll
                        for (int a = 0; a < NB; ++a) colb[buf + ty + 32 * a] = t[a][b];
                    }
            }
            __syncthreads();
            float piv = rowb[buf + k];
            if (!(piv > 0.0f)) {
                if (first_bad == 0) first_bad = q + 1;
                piv = 1.0f;
            }
            const float pinv = 1.0f / piv;
            // every entry: t_ij - t_ik t_kj / t_kk; row k and column k are
            // then overwritten by their owners
#pragma unroll
            for (int a = 0; a < NB; ++a) {
                const float ci = colb[buf + ty + 32 * a] * pinv;
#pragma unroll
                for (int b = 0; b < NB; ++b) t[a][b] = fmaf(-ci, rowb[buf + tx + 32 * b], t[a][b]);
            }
            if (ty == kl) {
#pragma unroll
                for (int a = 0; a < NB; ++a)
                    if (a == ka) {
#pragma unroll
                        for (int b = 0; b < NB; ++b) {
                            const int j = tx + 32 * b;
                            t[a][b] = (j == k) ? pinv : rowb[buf + j] * pinv;
                        }
                    }
            }
            if (tx == kl) {
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    if (b == ka) {
#pragma unroll
                        for (int a = 0; a < NB; ++a) {
                            const int i = ty + 32 * a;
                            if (i != k) t[a][b] = -colb[buf + i] * pinv;
                        }
                    }
            }
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < NB; ++a)
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int r = ty + 32 * a, c = tx + 32 * b;
                Dq[(size_t)r * B + c] = t[a][b];
                X[r * LD + c] = t[a][b];
            }
    }
    if (tid == 0) *flag = first_bad;
}

// G_q = T_q^-1 F_q stored column-major for the sweep:
// GT[c][r] = G[r][c] = sum_k F[k][c] Tinv[k][r] (T_q^-1 is symmetric); one
// CTA per block q >= 1.
template <int NB>
__global__ void __launch_bounds__(SPC_NT, 1) k_spc_gmul(const float* DF, float* G, int nb)
{
    constexpr int B = 32 * NB, LD = B + 1;
    extern __shared__ float smem[];
    float* As = smem;         // [32][LD]  F rows k0..k0+31
    float* Bs = As + 32 * LD; // [32][LD]  Tinv rows k0..k0+31
    const int q = blockIdx.x + 1;
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const size_t BB = (size_t)B * B;
    const float* Ti = DF + (size_t)q * BB;
    const float* FTq = DF + (size_t)nb * BB + (size_t)q * BB;
    float g[NB][NB];
#pragma unroll
    for (int a = 0; a < NB; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) g[a][b] = 0.0f;
    for (int k0 = 0; k0 < B; k0 += 32) {
        __syncthreads();
        for (int u = tid; u < 32 * B; u += SPC_NT) {
            const int c = u % B, kk = u / B;
            Bs[kk * LD + c] = Ti[(size_t)(k0 + kk) * B + c];
            const int kt = u & 31, ct = u >> 5;     // F[k][c] = FT[c][k], read along k
            As[kt * LD + ct] = FTq[(size_t)ct * B + k0 + kt];
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 32; ++kk) {
            float av[NB], bv[NB];
#pragma unroll
            for (int a = 0; a < NB; ++a) av[a] = As[kk * LD + ty + 32 * a];
#pragma unroll
            for (int b = 0; b < NB; ++b) bv[b] = Bs[kk * LD + tx + 32 * b];
#pragma unroll
            for (int a = 0; a < NB; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) g[a][b] = fmaf(av[a], bv[b], g[a][b]);
        }
    }
    float* Gq = G + (size_t)q * BB;
#pragma unroll
    for (int a = 0; a < NB; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) Gq[(size_t)(ty + 32 * a) * B + tx + 32 * b] = g[a][b];
}

// u_q = T_q^-1 r_q on the permuted residual (FP32), one CTA per block.
template <int NB>
__global__ void __launch_bounds__(SPC_NT) k_spc_u(const float* __restrict__ DF, const int* __restrict__ perm,
                                                 const cd* __restrict__ r, cf* __restrict__ h,
                                                 const CGState* __restrict__ st)
{
    constexpr int B = 32 * NB;
    __shared__ cf rv[B];
    if (st->done) return;
    const int q = blockIdx.x;
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    if (tid < B) {
        const int e = perm[q * B + tid];
        const cd v = e >= 0 ? r[e] : cd{0.0, 0.0};
        rv[tid] = cf{(float)v.x, (float)v.y};
    }
    __syncthreads();
    const float* Ti = DF + (size_t)q * B * B;
#pragma unroll
    for (int a = 0; a < NB; ++a) {
        const int row = ty + 32 * a;
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const float m = Ti[(size_t)row * B + tx + 32 * b];
            const cf x = rv[tx + 32 * b];
            sx = fmaf(m, x.x, sx);
            sy = fmaf(m, x.y, sy);
        }
        sx = warp_allsum_f(sx);
        sy = warp_allsum_f(sy);
        if (tx == 0) h[q * B + row] = cf{sx, sy};
    }
}

// The two sequential sweeps and the scatter back to element order.  The
// blocks are read column-major (MT[c][r]); warp g of the 16 owns the column
// slice [g B/16, (g+1) B/16) and lane l the rows [l NB, l NB + NB), so every
// load is a contiguous NB-float run of a column (coalesced across the warp)
// and the next block's slice is prefetched into registers while the
// current one is used.  The 16 partial sums of a row meet in shared memory.
constexpr int SW_NT = 512, SW_G = SW_NT / 32;

template <int NB>
__device__ __forceinline__ void load_run(const float* __restrict__ p, float (&d)[NB])
{
    if constexpr (NB == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
    } else if constexpr (NB == 2) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        d[0] = v.x;
        d[1] = v.y;
    } else {
#pragma unroll
        for (int i = 0; i < NB; ++i) d[i] = p[i];
    }
}

//
// With segs, CTA b sweeps the blocks segs[b].x .. segs[b].y of h in place
// (a segment's interior); with perm, the result is scattered to z in element
// order (the single chain).
template <int NB>
__global__ void __launch_bounds__(SW_NT, 1) k_spc_sweep(const float* __restrict__ Gm, const float* __restrict__ Hm,
                                                       const int* __restrict__ perm, cf* h, cd* __restrict__ z,
                                                       int nb, const CGState* __restrict__ st,
                                                       const int2* __restrict__ segs)
{
    constexpr int B = 32 * NB, CPW = B / SW_G;   // columns per warp
    __shared__ cf v[B];
    __shared__ cf part[SW_G][B];
    if (st->done) return;
    const int tid = threadIdx.x, lane = tid & 31, g = tid >> 5;
    const size_t BB = (size_t)B * B;
    const int r0 = lane * NB, cbase = g * CPW;
    float m[CPW][NB], mn[CPW][NB];
    cf un = cf{0.0f, 0.0f};
    auto load_blk = [&](const float* base, float (&dst)[CPW][NB]) {
#pragma unroll
        for (int j = 0; j < CPW; ++j) load_run<NB>(base + (size_t)(cbase + j) * B + r0, dst[j]);
    };
    // one step: y = u - M x, with x in v; y replaces v and h_q
    auto step = [&](int q, const cf u) {
        float px[NB], py[NB];
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            px[i] = 0.0f;
            py[i] = 0.0f;
        }
#pragma unroll
        for (int j = 0; j < CPW; ++j) {
            const cf x = v[cbase + j];
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                px[i] = fmaf(m[j][i], x.x, px[i]);
                py[i] = fmaf(m[j][i], x.y, py[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < NB; ++i) part[g][r0 + i] = cf{px[i], py[i]};
        __syncthreads();
        if (tid < B) {
            float sx = u.x, sy = u.y;
#pragma unroll
            for (int w = 0; w < SW_G; ++w) {
                const cf pw = part[w][tid];
                sx -= pw.x;
                sy -= pw.y;
            }
            const cf y = cf{sx, sy};
            v[tid] = y;
            h[(size_t)q * B + tid] = y;
        }
        __syncthreads();
    };
    const int2 sg = segs ? segs[blockIdx.x] : make_int2(0, nb - 1);
    const int qs = sg.x, qe = sg.y;
    if (tid < B) v[tid] = h[(size_t)qs * B + tid];
    // forward: h_q = u_q - G_q h_{q-1}
    if (qe > qs) {
        load_blk(Gm + (size_t)(qs + 1) * BB, mn);
        if (tid < B) un = h[(size_t)(qs + 1) * B + tid];
    }
    __syncthreads();
    for (int q = qs + 1; q <= qe; ++q) {
        const cf u = un;
#pragma unroll
        for (int j = 0; j < CPW; ++j)
#pragma unroll
            for (int i = 0; i < NB; ++i) m[j][i] = mn[j][i];
        if (q + 1 <= qe) {
            load_blk(Gm + (size_t)(q + 1) * BB, mn);
            if (tid < B) un = h[(size_t)(q + 1) * B + tid];
        }
        step(q, u);
    }
    // backward: x_q = h_q - H_q x_{q+1}; v holds x_qe = h_qe
    if (qe > qs) {
        load_blk(Hm + (size_t)(qe - 1) * BB, mn);
        if (tid < B) un = h[(size_t)(qe - 1) * B + tid];
    }
    for (int q = qe - 1; q >= qs; --q) {
        const cf u = un;
#pragma unroll
        for (int j = 0; j < CPW; ++j)
#pragma unroll
            for (int i = 0; i < NB; ++i) m[j][i] = mn[j][i];
        if (q > qs) {
            load_blk(Hm + (size_t)(q - 1) * BB, mn);
            if (tid < B) un = h[(size_t)(q - 1) * B + tid];
        }
        step(q, u);
    }
    if (!perm) return;
    for (int pos = tid; pos < nb * B; pos += SW_NT) {
        const int e = perm[pos];
        if (e >= 0) {
            const cf x = h[pos];
            z[e] = cd{(double)x.x, (double)x.y};
        }
    }
}

// ---------------------------------------------------------------------------
// Segmented form: block products on one CTA of (B/8)^2 threads, the layout of
// k_spc_factor_v (thread (ty, tx): rows 8 ty .. 8 ty + 7, column quads
// 4 tx .. and B/2 + 4 tx ..).  Operands are staged in shared memory as k-rows,
// At[k][r] = A[r][k] and Bk[k][c] = B[k][c], with the row stride B + 4.
template <int NB>
struct BlkMM {
    static constexpr int B = 32 * NB, TPR = B / 8, NT = TPR * TPR, HB = B / 2, LDS = B + 4;
    int tid, r0, c0;
    __device__ BlkMM() : tid(threadIdx.x), r0(8 * (threadIdx.x / TPR)), c0(4 * (threadIdx.x % TPR)) {}
    __device__ int col(int b) const { return (b >> 2) * HB + c0 + (b & 3); }
    // dst[k][j] = src[k][j] (src row-major B x B in global memory)
    __device__ void stage(float* dst, const float* __restrict__ src) const
    {
        for (int i = tid; i < B * B / 4; i += NT) {
            const int k = (4 * i) / B, j = (4 * i) % B;
            cp_async16(dst + k * LDS + j, src + 4 * (size_t)i);
        }
        cp_async_commit();
    }
    // dst[k][j] = src[j][k]
    __device__ void stage_t(float* dst, const float* __restrict__ src) const
    {
        for (int i = tid; i < B * B; i += NT) {
            const int j = i / B, k = i % B;
            dst[k * LDS + j] = src[i];
        }
    }
    // acc (+)= sum_k At[k][r] Bk[k][c]
    __device__ void mma(const float* At, const float* Bk, float (&acc)[8][8]) const
    {
#pragma unroll 2
        for (int k = 0; k < B; ++k) {
            const float4 a0 = *reinterpret_cast<const float4*>(At + k * LDS + r0);
            const float4 a1 = *reinterpret_cast<const float4*>(At + k * LDS + r0 + 4);
            const float4 b0 = *reinterpret_cast<const float4*>(Bk + k * LDS + c0);
            const float4 b1 = *reinterpret_cast<const float4*>(Bk + k * LDS + HB + c0);
            const float xa[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float xb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(xa[a], xb[b], acc[a][b]);
        }
    }
    __device__ void zero(float (&acc)[8][8]) const
    {
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = 0.0f;
    }
    // C row-major in global memory (ld B): load / store this thread's entries
    __device__ void load(const float* __restrict__ C, float (&v)[8][8]) const
    {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const float4 x = *reinterpret_cast<const float4*>(C + (size_t)(r0 + a) * B + c0);
            const float4 y = *reinterpret_cast<const float4*>(C + (size_t)(r0 + a) * B + HB + c0);
            v[a][0] = x.x; v[a][1] = x.y; v[a][2] = x.z; v[a][3] = x.w;
            v[a][4] = y.x; v[a][5] = y.y; v[a][6] = y.z; v[a][7] = y.w;
        }
    }
    __device__ void store(float* C, const float (&v)[8][8]) const
    {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            *reinterpret_cast<float4*>(C + (size_t)(r0 + a) * B + c0) = make_float4(v[a][0], v[a][1], v[a][2], v[a][3]);
            *reinterpret_cast<float4*>(C + (size_t)(r0 + a) * B + HB + c0) = make_float4(v[a][4], v[a][5], v[a][6], v[a][7]);
        }
    }
    // into shared memory as k-rows (row stride LDS) for the next product
    __device__ void store_s(float* Cs, const float (&v)[8][8]) const
    {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            *reinterpret_cast<float4*>(Cs + (r0 + a) * LDS + c0) = make_float4(v[a][0], v[a][1], v[a][2], v[a][3]);
            *reinterpret_cast<float4*>(Cs + (r0 + a) * LDS + HB + c0) = make_float4(v[a][4], v[a][5], v[a][6], v[a][7]);
        }
    }
    // C^T row-major in global memory (the F^T layout of DF)
    __device__ void store_t(float* C, const float (&v)[8][8]) const
    {
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            float* p = C + (size_t)col(b) * B + r0;
            *reinterpret_cast<float4*>(p) = make_float4(v[0][b], v[1][b], v[2][b], v[3][b]);
            *reinterpret_cast<float4*>(p + 4) = make_float4(v[4][b], v[5][b], v[6][b], v[7][b]);
        }
    }
};

template <int NB>
constexpr size_t spike_smem() { return sizeof(float) * 2 * (size_t)(32 * NB) * (32 * NB + 4); }

// The spikes of segment p (CTA 2p: V_p, CTA 2p + 1: W_p), from the segment
// factor (T_q^-1 in DF, G and H column-major):
//   V: X_s = T_s^-1 F_s, X_q = -G_q X_{q-1};  V[ie] = X_ie, V[q] = X_q - H_q V[q+1]
//   W: W[ie] = T_ie^-1 F_e^T,  W[q] = -H_q W[q+1]
// (s, ie the segment's first and last interior blocks, e its separator).
template <int NB>
__global__ void __launch_bounds__(16 * NB * NB, 1) k_spc_spike(const float* __restrict__ DF, const float* __restrict__ Gm,
                                                              const float* __restrict__ Hm, const int2* __restrict__ segs,
                                                              int nseg, int nb, float* V, float* W)
{
    using M = BlkMM<NB>;
    constexpr int B = M::B, LDS = M::LDS;
    extern __shared__ __align__(16) float smem[];
    float* At = smem;
    float* Bk = smem + B * LDS;
    const M mm;
    const int p = blockIdx.x >> 1, right = blockIdx.x & 1;
    if (right ? p >= nseg - 1 : p == 0) return;
    const int s = segs[p].x, ie = segs[p].y;
    const size_t BB = (size_t)B * B;
    const float* FT = DF + (size_t)nb * BB;
    float acc[8][8];
    if (!right) {
        // X_s = T_s^-1 F_s: At = T_s^-1 (symmetric), Bk[k][c] = F_s[k][c] = FT_s[c][k]
        mm.stage(At, DF + (size_t)s * BB);
        mm.stage_t(Bk, FT + (size_t)s * BB);
        cp_async_wait_all();
        __syncthreads();
        mm.zero(acc);
        mm.mma(At, Bk, acc);
        mm.store(V + (size_t)s * BB, acc);
        for (int q = s + 1; q <= ie; ++q) {
            __syncthreads();                       // At / Bk of the last product are consumed
            mm.store_s(Bk, acc);                   // X_{q-1}
            mm.stage(At, Gm + (size_t)q * BB);     // At[k][r] = G_q[r][k] = GT_q[k][r]
            cp_async_wait_all();
            __syncthreads();
            mm.zero(acc);
            mm.mma(At, Bk, acc);
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = -acc[a][b];
            mm.store(V + (size_t)q * BB, acc);
        }
        // back: acc holds V[ie] = X_ie
        for (int q = ie - 1; q >= s; --q) {
            __syncthreads();
            mm.store_s(Bk, acc);                   // V[q+1]
            mm.stage(At, Hm + (size_t)q * BB);     // At[k][r] = H_q[r][k] = HT_q[k][r]
            cp_async_wait_all();
            __syncthreads();
            float x[8][8];
            mm.load(V + (size_t)q * BB, x);        // X_q
            mm.zero(acc);
            mm.mma(At, Bk, acc);
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = x[a][b] - acc[a][b];
            mm.store(V + (size_t)q * BB, acc);
        }
    } else {
        const int e = ie + 1;
        // W[ie] = T_ie^-1 F_e^T: Bk[k][c] = F_e^T[k][c] = FT_e[k][c]
        mm.stage(At, DF + (size_t)ie * BB);
        mm.stage(Bk, FT + (size_t)e * BB);
        cp_async_wait_all();
        __syncthreads();
        mm.zero(acc);
        mm.mma(At, Bk, acc);
        mm.store(W + (size_t)ie * BB, acc);
        for (int q = ie - 1; q >= s; --q) {
            __syncthreads();
            mm.store_s(Bk, acc);                   // W[q+1]
            mm.stage(At, Hm + (size_t)q * BB);
            cp_async_wait_all();
            __syncthreads();
            mm.zero(acc);
            mm.mma(At, Bk, acc);
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = -acc[a][b];
            mm.store(W + (size_t)q * BB, acc);
        }
    }
}

// The separators' Schur complement, one CTA per separator p (block e):
//   Sd_p = D_e - F_e W[e-1] - F_{e+1}^T V[e+1]     -> DFc[p]       (row-major)
//   So_p = -F_e V[e-1]  (p >= 1)                   -> DFc[nc + p]  as So_p^T
template <int NB>
__global__ void __launch_bounds__(16 * NB * NB, 1) k_spc_reduced(const float* __restrict__ DF,
                                                                const float* __restrict__ V,
                                                                const float* __restrict__ W,
                                                                const int* __restrict__ sep, int nc, int nb,
                                                                float* DFc)
{
    using M = BlkMM<NB>;
    constexpr int B = M::B, LDS = M::LDS;
    extern __shared__ __align__(16) float smem[];
    float* At = smem;
    float* Bk = smem + B * LDS;
    const M mm;
    const int p = blockIdx.x, e = sep[p];
    const size_t BB = (size_t)B * B;
    const float* FT = DF + (size_t)nb * BB;
    float acc[8][8], d[8][8];
    mm.load(DF + (size_t)e * BB, d);                    // D_e (the segment factors leave it)
    // F_e W[e-1]: At[k][r] = F_e[r][k] = FT_e[k][r]
    mm.stage(At, FT + (size_t)e * BB);
    mm.stage(Bk, W + (size_t)(e - 1) * BB);
    cp_async_wait_all();
    __syncthreads();
    mm.zero(acc);
    mm.mma(At, Bk, acc);
    __syncthreads();
    // F_{e+1}^T V[e+1]: At[k][r] = F_{e+1}[k][r] = FT_{e+1}[r][k]
    mm.stage_t(At, FT + (size_t)(e + 1) * BB);
    mm.stage(Bk, V + (size_t)(e + 1) * BB);
    cp_async_wait_all();
    __syncthreads();
    mm.mma(At, Bk, acc);
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) d[a][b] -= acc[a][b];
    mm.store(DFc + (size_t)p * BB, d);
    if (p == 0) return;
    __syncthreads();
    // So_p = -F_e V[e-1]
    mm.stage(At, FT + (size_t)e * BB);
    mm.stage(Bk, V + (size_t)(e - 1) * BB);
    cp_async_wait_all();
    __syncthreads();
    mm.zero(acc);
    mm.mma(At, Bk, acc);
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = -acc[a][b];
    mm.store_t(DFc + (size_t)(nc + p) * BB, acc);
}

// Separators' right-hand sides and their first step, one CTA (B threads) per
// separator p (block e):  g = r_e - F_e y[e-1] - F_{e+1}^T y[e+1],
// hc_p = Tc_p^-1 g  (Tc_p^-1 symmetric, in DFc[p] after the reduced factor).
template <int NB>
__global__ void __launch_bounds__(32 * NB) k_spc_sep_rhs(const float* __restrict__ DF, const float* __restrict__ DFc,
                                                        const int* __restrict__ sep, const int* __restrict__ perm,
                                                        const cd* __restrict__ r, const cf* __restrict__ h,
                                                        cf* __restrict__ hc, int nb, const CGState* __restrict__ st)
{
    constexpr int B = 32 * NB;
    __shared__ cf yl[B], yr[B], g[B];
    if (st->done) return;
    const int p = blockIdx.x, e = sep[p], t = threadIdx.x;
    const size_t BB = (size_t)B * B;
    const float* FTe = DF + (size_t)nb * BB + (size_t)e * BB;
    const float* FTn = DF + (size_t)nb * BB + (size_t)(e + 1) * BB;
    yl[t] = h[(size_t)(e - 1) * B + t];
    yr[t] = h[(size_t)(e + 1) * B + t];
    const int el = perm[(size_t)e * B + t];
    const cd rv = el >= 0 ? r[el] : cd{0.0, 0.0};
    __syncthreads();
    float sx = (float)rv.x, sy = (float)rv.y;
    for (int k = 0; k < B; ++k) {
        // (F_e y)_t = sum_k FT_e[k][t] y_k ;  (F_{e+1}^T y)_t = sum_k FT_{e+1}[t][k] y_k
        const float a = FTe[(size_t)k * B + t], b = FTn[(size_t)t * B + k];
        sx -= a * yl[k].x + b * yr[k].x;
        sy -= a * yl[k].y + b * yr[k].y;
    }
    g[t] = cf{sx, sy};
    __syncthreads();
    const float* Tc = DFc + (size_t)p * BB;
    float ux = 0.0f, uy = 0.0f;
    for (int k = 0; k < B; ++k) {
        const float m = Tc[(size_t)k * B + t];
        ux = fmaf(m, g[k].x, ux);
        uy = fmaf(m, g[k].y, uy);
    }
    hc[(size_t)p * B + t] = cf{ux, uy};
}

// x_q = y_q - V[q] x_{c_{p-1}} - W[q] x_{c_p} for the interior blocks of
// segment p, x = xc_p for separator p; scattered to z in element order.  One
// CTA (B threads) per block.
template <int NB>
__global__ void __launch_bounds__(32 * NB) k_spc_correct(const float* __restrict__ V, const float* __restrict__ W,
                                                        const int* __restrict__ bseg, const int* __restrict__ perm,
                                                        const cf* __restrict__ h, const cf* __restrict__ hc,
                                                        cd* __restrict__ z, int nseg, const CGState* __restrict__ st)
{
    constexpr int B = 32 * NB;
    __shared__ cf xl[B], xr[B];
    if (st->done) return;
    const int q = blockIdx.x, t = threadIdx.x, sp = bseg[q];
    const size_t BB = (size_t)B * B;
    cf x;
    if (sp < 0) {
        x = hc[(size_t)(-1 - sp) * B + t];
    } else {
        const bool left = sp > 0, rightc = sp < nseg - 1;
        xl[t] = left ? hc[(size_t)(sp - 1) * B + t] : cf{0.0f, 0.0f};
        xr[t] = rightc ? hc[(size_t)sp * B + t] : cf{0.0f, 0.0f};
        __syncthreads();
        x = h[(size_t)q * B + t];
        // thread t's row of V and W by 16-byte loads (a row is 16-byte
        // aligned: B floats from a 16-byte aligned base), its entries taken
        // in order
        const float4* Vq = reinterpret_cast<const float4*>(V + (size_t)q * BB + (size_t)t * B);
        const float4* Wq = reinterpret_cast<const float4*>(W + (size_t)q * BB + (size_t)t * B);
        auto row = [&](const float4* Rq, const cf* xv) {
#pragma unroll 4
            for (int k4 = 0; k4 < B / 4; ++k4) {
                const float4 v = Rq[k4];
                const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    x.x -= e[u] * xv[4 * k4 + u].x;
                    x.y -= e[u] * xv[4 * k4 + u].y;
                }
            }
        };
        if (left) row(Vq, xl);
        if (rightc) row(Wq, xr);
    }
    const int el = perm[(size_t)q * B + t];
    if (el >= 0) z[el] = cd{(double)x.x, (double)x.y};
}

size_t factor_smem(int B) { return sizeof(float) * ((size_t)B * (B + 1) + 32 * (B + 1) + 4 * B); }
size_t factor_v_smem(int B) { return sizeof(float) * (3 * (size_t)B * B + 4 * B); }
size_t gmul_smem(int B) { return sizeof(float) * (2 * 32 * (size_t)(B + 1)); }

template <int NB>
void factor_nb(const SpcPlan& P, cudaStream_t s)
{
    const int B = 32 * NB;
    const size_t fs = factor_smem(B), gs = gmul_smem(B);
    cudaMemsetAsync(P.d_flag, 0, sizeof(int), s);
    cudaFuncSetAttribute(k_spc_gmul<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gs);
    if constexpr (NB <= 4) {
        const size_t vs = factor_v_smem(B);
        cudaFuncSetAttribute(k_spc_factor_v<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vs);
        if (P.nseg > 0) {
            // segment interiors side by side, their spikes, the separators'
            // Schur complement and its factor
            constexpr size_t ss = spike_smem<NB>();
            k_spc_factor_v<NB><<<P.nseg, 16 * NB * NB, vs, s>>>(P.d_DF, P.d_H, P.nb, P.d_flag, P.d_seg);
            k_spc_gmul<NB><<<P.nb - 1, SPC_NT, gs, s>>>(P.d_DF, P.d_G, P.nb);
            cudaFuncSetAttribute(k_spc_spike<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss);
            k_spc_spike<NB><<<2 * P.nseg, 16 * NB * NB, ss, s>>>(P.d_DF, P.d_G, P.d_H, P.d_seg, P.nseg, P.nb,
                                                                  P.d_V, P.d_W);
            cudaFuncSetAttribute(k_spc_reduced<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss);
            k_spc_reduced<NB><<<P.nc, 16 * NB * NB, ss, s>>>(P.d_DF, P.d_V, P.d_W, P.d_sep, P.nc, P.nb, P.d_DFc);
            k_spc_factor_v<NB><<<1, 16 * NB * NB, vs, s>>>(P.d_DFc, P.d_Hc, P.nc, P.d_flag, nullptr);
            if (P.nc > 1) k_spc_gmul<NB><<<P.nc - 1, SPC_NT, gs, s>>>(P.d_DFc, P.d_Gc, P.nc);
            return;
        }
        k_spc_factor_v<NB><<<1, 16 * NB * NB, vs, s>>>(P.d_DF, P.d_H, P.nb, P.d_flag, nullptr);
    } else {
        cudaFuncSetAttribute(k_spc_factor<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fs);
        k_spc_factor<NB><<<1, SPC_NT, fs, s>>>(P.d_DF, P.d_H, P.nb, P.d_flag);
    }
    if (P.nb > 1) k_spc_gmul<NB><<<P.nb - 1, SPC_NT, gs, s>>>(P.d_DF, P.d_G, P.nb);
}

template <int NB>
void apply_nb(const SpcPlan& P, const cd* r, cd* z, const CGState* st, cudaStream_t s)
{
    k_spc_u<NB><<<P.nb, SPC_NT, 0, s>>>(P.d_DF, P.d_perm, r, P.d_h, st);
    if constexpr (NB <= 4) {
        if (P.nseg > 0) {
            k_spc_sweep<NB><<<P.nseg, SW_NT, 0, s>>>(P.d_G, P.d_H, nullptr, P.d_h, nullptr, P.nb, st, P.d_seg);
            k_spc_sep_rhs<NB><<<P.nc, 32 * NB, 0, s>>>(P.d_DF, P.d_DFc, P.d_sep, P.d_perm, r, P.d_h, P.d_hc, P.nb, st);
            k_spc_sweep<NB><<<1, SW_NT, 0, s>>>(P.d_Gc, P.d_Hc, nullptr, P.d_hc, nullptr, P.nc, st, nullptr);
            k_spc_correct<NB><<<P.nb, 32 * NB, 0, s>>>(P.d_V, P.d_W, P.d_bseg, P.d_perm, P.d_h, P.d_hc, z, P.nseg, st);
            return;
        }
    }
    k_spc_sweep<NB><<<1, SW_NT, 0, s>>>(P.d_G, P.d_H, P.d_perm, P.d_h, z, P.nb, st, nullptr);
}

template <typename T>
bool alloc(T** p, size_t n)
{
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess;
}

// Segments of the chain: about sqrt(nb) of them (the sequential work per
// application is ~ 2 nb / nseg + 2 nseg block steps), each of at least four
// blocks; the last block of every segment but the last is a separator.
void segment_layout(int nb, std::vector<int2>& seg, std::vector<int>& bseg, std::vector<int>& sep)
{
    int ns = (int)std::lround(std::sqrt((double)nb));
    ns = std::max(2, std::min(ns, nb / 4));
    seg.clear();
    sep.clear();
    bseg.assign(nb, 0);
    for (int p = 0; p < ns; ++p) {
        const int b0 = (int)((long long)nb * p / ns), b1 = (int)((long long)nb * (p + 1) / ns);   // [b0, b1)
        const bool last = p == ns - 1;
        const int ie = last ? b1 - 1 : b1 - 2;
        seg.push_back(make_int2(b0, ie));
        for (int q = b0; q <= ie; ++q) bseg[q] = p;
        if (!last) {
            sep.push_back(b1 - 1);
            bseg[b1 - 1] = -1 - p;
        }
    }
}

// Device buffers of the segmented form that every factor owns (spikes and
// the separators' system).
bool alloc_seg_factor(SpcPlan& P)
{
    const size_t BB = (size_t)P.B * P.B;
    return alloc(&P.d_V, P.nb * BB) && alloc(&P.d_W, P.nb * BB) && alloc(&P.d_DFc, 2 * (size_t)P.nc * BB) &&
           alloc(&P.d_Gc, P.nc * BB) && alloc(&P.d_Hc, P.nc * BB) && alloc(&P.d_hc, (size_t)P.nc * P.B);
}

void free_seg_factor(SpcPlan& P)
{
    cudaFree(P.d_V);
    cudaFree(P.d_W);
    cudaFree(P.d_DFc);
    cudaFree(P.d_Gc);
    cudaFree(P.d_Hc);
    cudaFree(P.d_hc);
    P.d_V = P.d_W = P.d_DFc = P.d_Gc = P.d_Hc = nullptr;
    P.d_hc = nullptr;
}


}  // namespace

extern "C" int32_t crt_rcm_order(int32_t n, const int32_t* xadj, const int32_t* adj, int32_t* order,
                                  int32_t* bandwidth)
{
    if (n < 1 || !xadj || !order) return CRT_ERR_ARG;
    if (xadj[0] != 0) return CRT_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (xadj[i + 1] < xadj[i]) return CRT_ERR_ARG;
    const int nadj = xadj[n];
    if (nadj > 0 && !adj) return CRT_ERR_ARG;
    for (int e = 0; e < nadj; ++e)
        if (adj[e] < 0 || adj[e] >= n) return CRT_ERR_ARG;
    std::vector<int> xa(xadj, xadj + n + 1), ad(adj, adj + nadj), ord;
    rcm_order(n, xa, ad, ord);
    std::vector<int> pos(n);
    for (int k = 0; k < n; ++k) {
        order[k] = ord[k];
        pos[ord[k]] = k;
    }
    if (bandwidth) {
        int bw = 0;
        for (int v = 0; v < n; ++v)
            for (int e = xa[v]; e < xa[v + 1]; ++e) bw = std::max(bw, std::abs(pos[v] - pos[ad[e]]));
        *bandwidth = bw;
    }
    return CRT_OK;
}

int spc_plan_build(SpcPlan& P, int M, int ltri, int nx, int nnb, const double* smatm, const int* nachbar,
                   std::string& why)
{
    spc_plan_free(P);
    P.M = M;
    // directed non-zero off-diagonal entries (i, j, smatm index) of R
    std::vector<int> ei, ej, es;
    auto add = [&](int i, int j, long long s) {
        if (j == i || smatm[s] == 0.0) return;
        ei.push_back(i);
        ej.push_back(j);
        es.push_back((int)s);
    };
    if (ltri == 0) {
        for (int i = 0; i < M; ++i) {
            if (i > 0) add(i, i - 1, (long long)M + i - 1);
            if (i < M - 1) add(i, i + 1, (long long)M + i);
            if (i >= nx) add(i, i - nx, 2LL * M + i - nx);
            if (i < M - nx) add(i, i + nx, 2LL * M + i);
        }
    } else {
        for (int k = 0; k < nnb; ++k)
            for (int i = 0; i < M; ++i) {
                const int id = nachbar[(size_t)k * M + i];
                if (id > 0) add(i, id - 1, (long long)k * M + i);
            }
    }
    const size_t ne = ei.size();
    // symmetric adjacency for the ordering
    std::vector<int> xadj(M + 1, 0), adj;
    for (size_t k = 0; k < ne; ++k) {
        xadj[ei[k] + 1]++;
        xadj[ej[k] + 1]++;
    }
    for (int i = 0; i < M; ++i) xadj[i + 1] += xadj[i];
    adj.resize(xadj[M]);
    {
        std::vector<int> fill(xadj.begin(), xadj.end() - 1);
        for (size_t k = 0; k < ne; ++k) {
            adj[fill[ei[k]]++] = ej[k];
            adj[fill[ej[k]]++] = ei[k];
        }
    }
    std::vector<int> order;
    rcm_order(M, xadj, adj, order);
    std::vector<int> pos(M);
    for (int k = 0; k < M; ++k) pos[order[k]] = k;
    int bw = 0;
    for (size_t k = 0; k < ne; ++k) bw = std::max(bw, std::abs(pos[ei[k]] - pos[ej[k]]));
    P.bw = bw;
    const int B = std::max(32, (bw + 31) / 32 * 32);
    if (B > SPC_MAX_B) {
        why = "regulariser bandwidth " + std::to_string(bw) + " after reverse Cuthill-McKee exceeds " +
              std::to_string(SPC_MAX_B) + "; the block preconditioner is not available for this mesh";
        return 0;
    }
    P.B = B;
    P.nb = (M + B - 1) / B;
    P.Mp = P.nb * B;
    const size_t BB = (size_t)B * B;
    std::vector<int> perm(P.Mp, -1);
    for (int k = 0; k < M; ++k) perm[k] = order[k];
    std::vector<int4> ent;
    ent.reserve(ne);
    for (size_t k = 0; k < ne; ++k) {
        const int pi = pos[ei[k]], pj = pos[ej[k]];
        const int qi = pi / B, qj = pj / B, ri = pi % B, rj = pj % B;
        size_t dst;
        if (qi == qj) dst = (size_t)qi * BB + (size_t)ri * B + rj;
        else if (qi == qj + 1) dst = (size_t)P.nb * BB + (size_t)qi * BB + (size_t)rj * B + ri;   // FT_q
        else continue;   // upper block: the transpose of an F entry
        ent.push_back(int4{(int)dst, ei[k], ej[k], es[k]});
    }
    P.nent = (int)ent.size();
    if (2 * (size_t)P.nb * BB > (size_t)INT32_MAX) {
        why = "block preconditioner too large for 32-bit entry offsets";
        return 0;
    }
    bool ok = alloc(&P.d_perm, P.Mp) && alloc(&P.d_ent, ent.size()) && alloc(&P.d_DF, 2 * P.nb * BB) &&
              alloc(&P.d_G, P.nb * BB) && alloc(&P.d_H, P.nb * BB) && alloc(&P.d_h, P.Mp) && alloc(&P.d_flag, 1);
    if (!ok) {
        spc_plan_free(P);
        return CRT_ERR_ALLOC;
    }
    if (cudaMemcpy(P.d_perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        (ent.size() && cudaMemcpy(P.d_ent, ent.data(), ent.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess)) {
        spc_plan_free(P);
        return CRT_ERR_CUDA;
    }
    // segmented form for B <= 128 and long chains (CRT_B200_SPC=single keeps
    // the single chain)
    const char* sv = std::getenv("CRT_B200_SPC");
    const bool single = sv && std::strcmp(sv, "single") == 0;
    if (!single && B <= 128 && P.nb >= 32) {
        std::vector<int2> seg;
        std::vector<int> bseg, sep;
        segment_layout(P.nb, seg, bseg, sep);
        P.nseg = (int)seg.size();
        P.nc = (int)sep.size();
        if (!alloc(&P.d_seg, seg.size()) || !alloc(&P.d_bseg, bseg.size()) || !alloc(&P.d_sep, sep.size()) ||
            !alloc_seg_factor(P)) {
            spc_plan_free(P);
            return CRT_ERR_ALLOC;
        }
        if (cudaMemcpy(P.d_seg, seg.data(), seg.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(P.d_bseg, bseg.data(), bseg.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(P.d_sep, sep.data(), sep.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
            spc_plan_free(P);
            return CRT_ERR_CUDA;
        }
    }
    P.ok = 1;
    return 0;
}

void spc_plan_free(SpcPlan& P)
{
    cudaFree(P.d_perm);
    cudaFree(P.d_ent);
    cudaFree(P.d_DF);
    cudaFree(P.d_G);
    cudaFree(P.d_H);
    cudaFree(P.d_h);
    cudaFree(P.d_flag);
    cudaFree(P.d_seg);
    cudaFree(P.d_bseg);
    cudaFree(P.d_sep);
    free_seg_factor(P);
    P = SpcPlan{};
}

int spc_plan_clone(const SpcPlan& src, SpcPlan& dst)
{
    spc_plan_free_clone(dst);
    if (!src.ok) return CRT_ERR_ARG;
    dst = src;   // ordering, entry list, segment layout and sizes are shared
    dst.ok = 0;
    dst.d_DF = nullptr;
    dst.d_G = dst.d_H = nullptr;
    dst.d_h = nullptr;
    dst.d_flag = nullptr;
    dst.d_V = dst.d_W = dst.d_DFc = dst.d_Gc = dst.d_Hc = nullptr;
    dst.d_hc = nullptr;
    const size_t BB = (size_t)src.B * src.B;
    const bool ok = alloc(&dst.d_DF, 2 * src.nb * BB) && alloc(&dst.d_G, src.nb * BB) &&
                    alloc(&dst.d_H, src.nb * BB) && alloc(&dst.d_h, src.Mp) && alloc(&dst.d_flag, 1) &&
                    (src.nseg == 0 || alloc_seg_factor(dst));
    if (!ok) {
        spc_plan_free_clone(dst);
        return CRT_ERR_ALLOC;
    }
    dst.ok = 1;
    return 0;
}

void spc_plan_free_clone(SpcPlan& P)
{
    cudaFree(P.d_DF);
    cudaFree(P.d_G);
    cudaFree(P.d_H);
    cudaFree(P.d_h);
    cudaFree(P.d_flag);
    free_seg_factor(P);
    P = SpcPlan{};
}

void launch_spc_factor(const SpcPlan& P, const double* cgfac, const double* smatm, double lam, cudaStream_t s)
{
    const size_t BB = (size_t)P.B * P.B;
    cudaMemsetAsync(P.d_DF, 0, 2 * P.nb * BB * sizeof(float), s);
    k_spc_diag<<<(P.nb * P.B + 255) / 256, 256, 0, s>>>(P.d_DF, P.nb, P.B);
    if (P.nent) k_spc_entries<<<(P.nent + 255) / 256, 256, 0, s>>>(P.d_ent, P.nent, cgfac, smatm, lam, P.d_DF);
    switch (P.B / 32) {
    case 1: factor_nb<1>(P, s); break;
    case 2: factor_nb<2>(P, s); break;
    case 3: factor_nb<3>(P, s); break;
    case 4: factor_nb<4>(P, s); break;
    case 5: factor_nb<5>(P, s); break;
    default: factor_nb<6>(P, s); break;
    }
}

void launch_spc_apply(const SpcPlan& P, const cd* r, cd* z, const CGState* st, cudaStream_t s)
{
    switch (P.B / 32) {
    case 1: apply_nb<1>(P, r, z, st, s); break;
    case 2: apply_nb<2>(P, r, z, st, s); break;
    case 3: apply_nb<3>(P, r, z, st, s); break;
    case 4: apply_nb<4>(P, r, z, st, s); break;
    case 5: apply_nb<5>(P, r, z, st, s); break;
    default: apply_nb<6>(P, r, z, st, s); break;
    }
}
