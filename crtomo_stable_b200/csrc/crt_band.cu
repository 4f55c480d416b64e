// crt_band.cu -- batched band Cholesky path of the forward model.
//
// One CTA owns one band system (one wavenumber k and, with mixed boundaries,
// one source electrode l).  The system is never materialised in HBM:
//
//   * rows of the FE matrix are formed when they enter an (mb+1)-row window
//     from the gather lists (kompab / kompadc, src/kompab.f90:80-128), with
//     the Dirichlet edits of randb / randb2 and the diagonal scaling of
//     scalab / scaldc (src/scalab.f90:52-76) applied on the way in;
//   * the window is factored right-looking, column by column (the same
//     L L^T, unconjugated for complex systems, as src/chol.f90:44-78), and the
//     system's own right-hand side is forward-substituted in the same pass
//     (the first half of src/vre.f90:45-56);
//   * each finished column of L leaves the window for a column-packed HBM
//     workspace; the back substitution (src/vre.f90:58-69) streams it back.
//
// The window is addressed in "slot space": row r lives in slot r mod W,
// W = mb + 1, and the symmetric entry of rows (r1, r2) sits at the packed
// index of the unordered slot pair, so a slot freed by the outgoing column
// is exactly the storage the incoming row needs.
#include "crt_band.h"

namespace {

__device__ __forceinline__ int pair_index(int x, int y)
{
    return x >= y ? x * (x + 1) / 2 + y : y * (y + 1) / 2 + x;
}

template <typename T>
__device__ __forceinline__ T assemble_entry(const BandArgs<T>& A, int e, int k, int l)
{
    T v = Sc<T>::zero();
    const int c1 = A.ent_ptr[e + 1];
    const double* elbg_k = A.elbg + (size_t)k * A.E * A.nmn;
    for (int c = A.ent_ptr[e]; c < c1; ++c) {
        const int code = A.con_code[c];
        double coef;
        if (code >= 0) {
            coef = elbg_k[code];
        } else {
            const int q = -code - 1;
            coef = A.relbg[q] * A.kg[((size_t)k * A.L + l) * A.R + q / 3];
        }
        v += scale(Sc<T>::from(A.sigma[A.con_sig[c]]), coef);
    }
    return v;
}

// Source vector entry of row r before scaling: kompab sets b(enr(l)) = -1
// and b(nsink) = +1, randb zeroes type-13 nodes, randb2 prescribes -value
// at boundary.dat nodes and moves their couplings (bdir) to the free rows.
template <typename T>
__device__ __forceinline__ T rhs_entry(int r, int src, int lsink, int nsink0,
                                       const unsigned char* dflag, const cd* dval, const cd* bdir)
{
    T b = Sc<T>::zero();
    if (r == src) b = -Sc<T>::one();
    if (lsink && r == nsink0) b = Sc<T>::one();
    const unsigned char f = dflag[r];
    if (f == 1) b = Sc<T>::zero();
    else if (f == 2) b = -Sc<T>::from(dval[r]);
    else if (bdir) b += Sc<T>::from(bdir[r]);
    return b;
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_band_factor(BandArgs<T> A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = A.W, n = A.n, mb = A.mb;
    const int P = W * (W + 1) / 2;
    T* win = reinterpret_cast<T*>(smem_raw);
    T* col = win + P;
    T* bsl = col + W;
    T* rowbuf = bsl + W;
    double* fakw = reinterpret_cast<double*>(rowbuf + W);
    __shared__ T s_piv;
    __shared__ double s_fak;
    __shared__ int s_err;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    const int b = blockIdx.x, sys = A.sys0 + b;
    int k, l;
    if (A.mixed) {
        k = sys / A.L;
        l = sys % A.L;
    } else {
        k = sys;
        l = 0;
    }
    T* Lc = A.Lws + (size_t)b * A.lstride;
    double* fk = A.fakws + (size_t)b * n;
    const bool fuse = A.fuse_rhs != 0;
    T* yv = fuse ? A.yws + (size_t)b * n : nullptr;
    const cd* bdir = (fuse && A.bdir) ? A.bdir + (size_t)b * n : nullptr;
    const int src = A.enr0[l];

    for (int i = tid; i < P; i += NT) win[i] = Sc<T>::zero();
    for (int i = tid; i < W; i += NT) {
        col[i] = Sc<T>::zero();
        bsl[i] = Sc<T>::zero();
        rowbuf[i] = Sc<T>::zero();
        fakw[i] = 0.0;
    }
    if (tid == 0) s_err = 0;
    __syncthreads();

    // Raw (unscaled) entries of row r into rowbuf[d].
    auto assemble_row = [&](int r) {
        const int e1 = A.row_ptr[r + 1];
        for (int e = A.row_ptr[r] + tid; e < e1; e += NT) rowbuf[A.ent_d[e]] = assemble_entry(A, e, k, l);
    };
    // Scaling factor of row r from its raw diagonal (thread 0).
    auto row_fak = [&](int r) {
        T raw = A.dflag[r] ? Sc<T>::one() : rowbuf[0];
        double d = Sc<T>::absval(raw);
        double f = 1.0;
        if (!(d > 0.0)) {
            s_err = CRT_ERR_ZERO_DIAG;
        } else {
            f = 1.0 / sqrt(d);
        }
        s_fak = f;
        fk[r] = f;
    };
    // Scaled row r into slot sr; clears rowbuf.
    auto scatter_row = [&](int r, int sr, double fr) {
        const bool dr = A.dflag[r] != 0;
        for (int d = tid; d <= mb; d += NT) {
            const int c = r - d;
            if (c < 0) continue;
            const int sc_ = c % W;
            T v;
            if (d == 0) {
                T raw = dr ? Sc<T>::one() : rowbuf[0];
                v = Sc<T>::normalise(raw, Sc<T>::absval(raw));
            } else {
                v = (dr || A.dflag[c]) ? Sc<T>::zero() : scale(rowbuf[d], fr * fakw[sc_]);
            }
            win[pair_index(sr, sc_)] = v;
            rowbuf[d] = Sc<T>::zero();
        }
        if (tid == 0) {
            fakw[sr] = fr;
            if (fuse) bsl[sr] = scale(rhs_entry<T>(r, src, A.lsink, A.nsink0, A.dflag, A.dval, bdir), fr);
        }
    };

    // Initial window: rows 0 .. W-1.
    const int r0n = min(W, n);
    for (int r = 0; r < r0n; ++r) {
        assemble_row(r);
        __syncthreads();
        if (tid == 0) row_fak(r);
        __syncthreads();
        scatter_row(r, r % W, s_fak);
        __syncthreads();
    }

    for (int i = 0; i < n; ++i) {
        const int s = i % W;
        const int rnew = i + W;
        // Phase A: pivot of column i, raw assembly of the incoming row.
        if (tid == 0) {
            T p = win[pair_index(s, s)];
            if (Sc<T>::bad_pivot(p)) s_err = CRT_ERR_PIVOT;
            T lii = Sc<T>::sqrt_(p);
            s_piv = lii;
            Lc[(size_t)i * W] = lii;
            if (fuse) {
                T yi = Sc<T>::div(bsl[s], lii);
                bsl[s] = yi;
                yv[i] = yi;
            }
        }
        if (rnew < n) assemble_row(rnew);
        __syncthreads();
        if (s_err) break;
        // Phase B: column i of L, forward substitution, scaling of the new row.
        {
            const T lii = s_piv;
            const T yi = fuse ? bsl[s] : Sc<T>::zero();
            for (int x = tid; x < W; x += NT) {
                if (x == s) continue;
                const int d = (x - s + W) % W;
                T v = Sc<T>::zero();
                if (i + d < n) v = Sc<T>::div(win[pair_index(x, s)], lii);
                col[x] = v;
                Lc[(size_t)i * W + d] = v;
                if (fuse) bsl[x] -= Sc<T>::mul(v, yi);
            }
            if (tid == 0) {
                col[s] = Sc<T>::zero();
                if (rnew < n) row_fak(rnew);
            }
        }
        __syncthreads();
        // Phase C: rank-1 update of the trailing window (slot s excluded),
        // and the new row into the freed slot s.
        for (int x = warp; x < W; x += NW) {
            if (x == s) continue;
            const int dx = (x - s + W) % W;
            if (i + dx >= n) continue;
            const T cx = col[x];
            T* wrow = win + x * (x + 1) / 2;
            for (int y = lane; y <= x; y += 32) {
                if (y == s) continue;
                wrow[y] -= Sc<T>::mul(cx, col[y]);
            }
        }
        if (rnew < n) scatter_row(rnew, s, s_fak);
        __syncthreads();
    }
    if (tid == 0) A.status[sys] = s_err;
}

// Back substitution (and, for systems without a fused forward pass, the
// forward substitution of the kompb right-hand side, src/kompb.f90:39-66).
// Both sweeps are blocked by BB columns: the off-block part of every column
// is a coalesced dot/axpy over the column-packed factor, the in-block
// triangle is solved by one warp.
template <typename T> __device__ __forceinline__ T shfl_idx_t(T v, int src);
template <> __device__ __forceinline__ double shfl_idx_t<double>(double v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}
template <> __device__ __forceinline__ cd shfl_idx_t<cd>(cd v, int src)
{
    return cd{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}
template <typename T> __device__ __forceinline__ T shfl_down_t(T v, int off);
template <> __device__ __forceinline__ double shfl_down_t<double>(double v, int off)
{
    return __shfl_down_sync(0xffffffffu, v, off);
}
template <> __device__ __forceinline__ cd shfl_down_t<cd>(cd v, int off)
{
    return cd{__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off)};
}
template <> __device__ __forceinline__ cf shfl_idx_t<cf>(cf v, int src)
{
    return cf{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}
template <> __device__ __forceinline__ cf shfl_down_t<cf>(cf v, int off)
{
    return cf{__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off)};
}

// Resident CTAs per SM of the solve (latency hiding across systems): two;
// complex64, whose prefetch double buffer of a 32-column block is 66.5 KB at
// mb = 129, three (the forward and backward triangles share one buffer).
template <typename T> struct SolveOcc { static constexpr int v = 2; };
template <> struct SolveOcc<cf> { static constexpr int v = 3; };
// complex64 solves stage the next block of 32 columns of the factor (one
// contiguous run: the factor is column-packed with an even column stride)
// in a shared double buffer, by one bulk copy, while the current block is
// solved
template <typename T> struct SolvePrefetch { static constexpr bool v = false; };
template <> struct SolvePrefetch<cf> { static constexpr bool v = true; };

template <typename T, int NT, int BB>
__global__ void __launch_bounds__(NT, NT == 128 ? 2 * SolveOcc<T>::v : SolveOcc<T>::v)
    k_band_solve(SolveArgs<T> A, T* scratch)
{
    // the forward pass's triangle tri[c][d] and the backward pass's trw[r][c]
    // share one buffer (the passes are separated by a barrier)
    __shared__ __align__(16) T trbuf[BB * (BB + 1)];
    T(*tri)[BB] = reinterpret_cast<T(*)[BB]>(trbuf);
    __shared__ T part[BB];
    __shared__ T zb[BB];
    extern __shared__ __align__(16) unsigned char solve_dyn[];
    T* lbuf = reinterpret_cast<T*>(solve_dyn);   // [2][BB * W] (prefetching form)
    constexpr bool PF = SolvePrefetch<T>::v;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = A.n, W = A.W, mb = A.mb;
    const int b = blockIdx.x, sys = A.sys0 + b;
    // a refinement correction of a system already at the FP64 floor is skipped
    // (uniform over the CTA, before any barrier)
    if (A.skip_omega && refine_done(A.skip_omega, b, A.skip_tau)) return;
    const int slot = b / A.factor_of_sys_div;
    // solve systems are always (k, l) pairs, sys = k * L + l
    const int k = sys / A.L, l = sys % A.L;
    const T* Lc = A.Lws + (size_t)slot * A.lstride;
    const double* fk = A.fakws + (size_t)slot * n;
    T* z = scratch + (size_t)b * n;
    // columns [c0, c0 + nb) of the factor into buffer `buf` by one bulk
    // copy (TMA engine) completing on the buffer's mbarrier; pf_wait(buf)
    // returns once it has landed (bounded: a timeout marks the system)
    __shared__ __align__(8) unsigned long long pbar[2];
    int pphase[2] = {0, 0};
    if (PF && tid == 0) {
        mbar_init(&pbar[0], 1);
        mbar_init(&pbar[1], 1);
    }
    auto prefetch = [&](int c0, int nb, int buf) {
        if (tid == 0) {
            const int bytes = nb * W * (int)sizeof(T);
            mbar_expect_tx(&pbar[buf], bytes);
            bulk_g2s(lbuf + (size_t)buf * BB * W, Lc + (size_t)c0 * W, bytes, &pbar[buf]);
        }
    };
    auto pf_wait = [&](int buf) {
        if (!mbar_wait(&pbar[buf], pphase[buf])) A.status[sys] = CRT_ERR_CUDA;
        pphase[buf] ^= 1;
    };

    // The fused forward pass belongs to the system's own right-hand side:
    // every (k, l) system with mixed boundaries, only electrode 1 otherwise
    // (the reference refactors for l == 1 and calls kompb for l > 1).  An
    // explicit right-hand side (the refinement's residual) is solved in full.
    const bool use_fused = A.yws && !A.rhs && (A.mixed || l == 0);
    if (use_fused) {
        const T* y = A.yws + (size_t)slot * n;
        for (int i = tid; i < n; i += NT) z[i] = y[i];
    } else {
        if (A.rhs) {
            const T* rb = A.rhs + (size_t)b * n;
            for (int i = tid; i < n; i += NT) z[i] = rb[i];
        } else {
            // kompb right-hand side: b(enr(l)) = -fak, b(nsink) = +fak.
            for (int i = tid; i < n; i += NT) z[i] = Sc<T>::zero();
            __syncthreads();
            if (tid == 0) {
                const int src = A.enr0[l];
                z[src] = scale(-Sc<T>::one(), fk[src]);
                if (A.lsink) z[A.nsink0] = scale(Sc<T>::one(), fk[A.nsink0]);
            }
        }
        if (tid < BB) zb[tid] = Sc<T>::zero();
        __syncthreads();
        // Forward substitution L y = b by blocks of BB rows: the block's
        // triangle is staged by columns and solved by warp 0 with one unknown
        // per lane (reciprocal pivots, one shuffle broadcast per unknown);
        // the following mb rows then take the block's columns right-looking
        // (coalesced over the rows of a column).
        if constexpr (PF) {
            prefetch(0, min(n, BB), 0);
            pf_wait(0);
            __syncthreads();
        }
        int fbuf = 0;
        for (int c0 = 0; c0 < n; c0 += BB) {
            const int c1 = min(n, c0 + BB), nb = c1 - c0;
            const T* blk = PF ? lbuf + (size_t)fbuf * BB * W : Lc + (size_t)c0 * W;   // column c0 + cc at cc * W
            if constexpr (PF) {
                if (c1 < n) prefetch(c1, min(n, c1 + BB) - c1, fbuf ^ 1);
            }
            for (int t = tid; t < BB * BB; t += NT) {
                const int cc = t / BB, d = t % BB;
                tri[cc][d] = (cc < nb && d <= mb && cc + d < nb) ? blk[(size_t)cc * W + d] : Sc<T>::zero();
            }
            __syncthreads();
            if (warp == 0) {
                T v = Sc<T>::zero(), dinv = Sc<T>::zero();
                if (lane < nb) {
                    v = z[c0 + lane];
                    dinv = Sc<T>::recip(tri[lane][0]);
                }
                for (int cc = 0; cc < nb; ++cc) {
                    if (lane == cc) v = Sc<T>::mul(v, dinv);
                    const T y = shfl_idx_t(v, cc);
                    if (lane > cc && lane < nb) v -= Sc<T>::mul(tri[cc][lane - cc], y);
                }
                if (lane < nb) {
                    z[c0 + lane] = v;
                    zb[lane] = v;
                }
            }
            __syncthreads();
            // rows beyond the block: b_r -= sum_c L(r, c) y_c, eight columns'
            // loads in flight at a time (coalesced over the rows of a column)
            for (int r = c1 + tid; r < min(n, c1 + mb); r += NT) {
                const int cc0 = max(0, r - mb - c0);
                T acc = Sc<T>::zero();
                for (int cb = 0; cb < BB; cb += 8) {
                    T lv[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int cc = cb + u;
                        lv[u] = (cc >= cc0 && cc < nb) ? blk[(size_t)cc * W + (r - c0 - cc)] : Sc<T>::zero();
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) acc += Sc<T>::mul(lv[u], zb[cb + u]);
                }
                z[r] -= acc;
            }
            if constexpr (PF) {
                if (c1 < n) pf_wait(fbuf ^ 1);
                // the buffer just read is the next bulk copy's destination
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            }
            __syncthreads();
            fbuf ^= 1;
        }
    }
    __syncthreads();
    // Back substitution L^T x = y, blocked from the end.  Per block of BB
    // columns, NT/BB consecutive threads own a column: they keep all loads
    // of its off-block part in flight for the dot product with the solved
    // unknowns and stage its in-block entries row-wise (zeros beyond the
    // band, so no entry of an earlier block survives); one warp then
    // solves the BB x BB triangle with one unknown per lane (the pivots'
    // reciprocals are formed off the critical path, and each unknown costs
    // one shuffle broadcast and one FMA per lane).
    constexpr int TPC = NT / BB;
    static_assert(BB == 32 && TPC * BB == NT && (TPC & (TPC - 1)) == 0, "solve layout");
    T(*trw)[BB + 1] = reinterpret_cast<T(*)[BB + 1]>(trbuf);   // trw[r][c] = L(c0 + r, c0 + c), r >= c
    const int col = tid / TPC, sub = tid % TPC;
    if constexpr (PF) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        prefetch(max(0, n - BB), n - max(0, n - BB), 0);
        pf_wait(0);
        __syncthreads();
    }
    int bbuf = 0;
    for (int c1 = n; c1 > 0; c1 -= BB) {
        const int c0 = max(0, c1 - BB), nb = c1 - c0;
        if constexpr (PF) {
            if (c0 > 0) prefetch(max(0, c0 - BB), c0 - max(0, c0 - BB), bbuf ^ 1);
        }
        T acc = Sc<T>::zero();
        if (col < nb) {
            const int c = c0 + col;
            const T* Lcol = PF ? lbuf + (size_t)bbuf * BB * W + (size_t)col * W : Lc + (size_t)c * W;
            const int dmax = min(mb, n - 1 - c);
            const int din = nb - col;          // d < din: rows inside the block
            const int dend = max(dmax, din - 1);
#pragma unroll 8
            for (int d = sub; d <= dend; d += TPC) {
                const T v = d <= dmax ? Lcol[d] : Sc<T>::zero();
                if (d < din) trw[col + d][col] = v;
                else acc += Sc<T>::mul(v, z[c + d]);
            }
        }
#pragma unroll
        for (int off = TPC / 2; off > 0; off >>= 1) acc += shfl_down_t(acc, off);
        if (sub == 0 && col < nb) part[col] = acc;
        __syncthreads();
        if (warp == 0) {
            T v = Sc<T>::zero(), dinv = Sc<T>::zero();
            if (lane < nb) {
                v = z[c0 + lane] - part[lane];
                dinv = Sc<T>::recip(trw[lane][lane]);
            }
            for (int cc = nb - 1; cc >= 0; --cc) {
                if (lane == cc) v = Sc<T>::mul(v, dinv);
                const T x = shfl_idx_t(v, cc);
                if (lane < cc) v -= Sc<T>::mul(trw[cc][lane], x);
            }
            if (lane < nb) z[c0 + lane] = v;
        }
        if constexpr (PF) {
            if (c0 > 0) pf_wait(bbuf ^ 1);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        }
        __syncthreads();
        bbuf ^= 1;
    }
    // kpot(j, l, k) = pot(j) * fak(j) with pot = -z (a refinement step adds
    // the correction's contribution).
    cd* out = A.kpot + ((size_t)k * A.L + l) * n;
    if (A.accumulate) {
        for (int j = tid; j < n; j += NT) out[j] = out[j] - Sc<T>::to_cd(z[j]) * fk[j];
    } else {
        for (int j = tid; j < n; j += NT) out[j] = Sc<T>::to_cd(scale(-z[j], fk[j]));
    }
    (void)A.status;
}

}  // namespace

template <typename T>
size_t band_factor_smem(int W)
{
    size_t P = (size_t)W * (W + 1) / 2;
    return P * sizeof(T) + 3 * (size_t)W * sizeof(T) + (size_t)W * sizeof(double) + 64;
}

template <typename T>
void launch_band_factor(const BandArgs<T>& a, cudaStream_t st)
{
    constexpr int NT = 256;
    size_t smem = band_factor_smem<T>(a.W);
    cudaFuncSetAttribute(k_band_factor<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_band_factor<T, NT><<<a.nsys, NT, smem, st>>>(a);
}

// The solve kernel needs one n-vector of scratch per system; it is carved
// from the caller's y workspace when the forward pass was fused, otherwise
// from a dedicated buffer passed through SolveArgs::yws == NULL.
template <typename T>
void launch_band_solve_with_scratch(const SolveArgs<T>& a, T* scratch, cudaStream_t st)
{
    constexpr int BB = 32;
    size_t dyn = 0;
    if (SolvePrefetch<T>::v) dyn = 2 * (size_t)BB * a.W * sizeof(T);
    auto go = [&](auto kern, int nt) {
        if (dyn) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        }
        kern<<<a.nsys, nt, dyn, st>>>(a, scratch);
    };
    // narrow bands: a column has few entries, so half the threads per CTA
    // and twice the CTAs per SM hide more of the per-block latency
    if (a.W <= 80) go(k_band_solve<T, 128, BB>, 128);
    else go(k_band_solve<T, 256, BB>, 256);
}

template size_t band_factor_smem<double>(int);
template size_t band_factor_smem<cd>(int);
template void launch_band_factor<double>(const BandArgs<double>&, cudaStream_t);
template void launch_band_factor<cd>(const BandArgs<cd>&, cudaStream_t);
template void launch_band_solve_with_scratch<double>(const SolveArgs<double>&, double*, cudaStream_t);
template void launch_band_solve_with_scratch<cd>(const SolveArgs<cd>&, cd*, cudaStream_t);
template void launch_band_solve_with_scratch<cf>(const SolveArgs<cf>&, cf*, cudaStream_t);
