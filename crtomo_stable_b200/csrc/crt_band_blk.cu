// crt_band_blk.cu -- panel-blocked band factorisation (the production
// variant of k_band_factor, same inputs, outputs and arithmetic contract).
//
// One CTA per band system.  The window holds Wn = roundup(mb + PB, PB) rows
// in shared memory; row r lives in slot r mod Wn and the symmetric entry of
// two rows is stored once, at the unordered slot pair, in 4 x 4 tiles
// (tile (X, Y), X >= Y, row-major inside the tile).  Per panel of PB
// columns [i0, i0 + PB):
//   1. warp 0 factors the PB x PB diagonal block (unconjugated L L^T, the
//      recurrence of src/chol.f90:44-78 restricted to the block) and
//      forward-substitutes the panel's right-hand side; warps 1.. form the
//      next PB rows from the gather lists (kompab) into a staging buffer;
//   2. every window row below the panel solves its PB entries against the
//      block (L_x = A_x L_D^-T), updates its right-hand side and writes its
//      L entries to the window and to the column-packed HBM factor;
//   3. the trailing window is updated by the rank-PB product L_x L_y^T, each
//      thread accumulating 4 x 4 tiles in registers;
//   4. the PB staged rows are scaled (scalab), Dirichlet-edited (randb) and
//      written into the slots the panel freed.
// Four CTA barriers per PB columns replace the three per column of the
// rank-1 variant.
#include "crt_band.h"

namespace {

constexpr int TILE = 4;
// Tiles are stored 17 elements apart (16 used): consecutive tiles then start
// in consecutive 16-byte bank groups, so the per-thread tile accesses of a
// warp do not collide in shared memory.
constexpr int TSTRIDE = 17;

__device__ __forceinline__ int tile_base(int X, int Y) { return ((X * (X + 1)) >> 1) + Y; }

// Packed index of the unordered slot pair {x, y}.
__device__ __forceinline__ int widx(int x, int y)
{
    if (x < y) {
        int t = x;
        x = y;
        y = t;
    }
    return tile_base(x >> 2, y >> 2) * TSTRIDE + ((x & 3) << 2) + (y & 3);
}

template <typename T>
__device__ __forceinline__ T shfl_T(T v, int src);
template <>
__device__ __forceinline__ double shfl_T<double>(double v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}
template <>
__device__ __forceinline__ cd shfl_T<cd>(cd v, int src)
{
    return cd{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}

template <typename T>
__device__ __forceinline__ T assemble_entry_b(const BandArgs<T>& A, int e, int k, int l)
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

template <typename T>
__device__ __forceinline__ T rhs_entry_b(int r, int src, int lsink, int nsink0, const unsigned char* dflag,
                                         const cd* dval, const cd* bdir)
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

template <typename T, int PB, int NT>
__global__ void __launch_bounds__(NT) k_band_factor_blk(BandArgs<T> A, int Wn)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = A.n, mb = A.mb, W1 = A.W;    // W1 = mb + 1 (column stride of the HBM factor)
    const int NTR = Wn / TILE;
    const int NTT = NTR * (NTR + 1) / 2;
    T* win = reinterpret_cast<T*>(smem_raw);              // NTT * TSTRIDE
    T* stage = win + (size_t)NTT * TSTRIDE;               // PB * W1
    T* LD = stage + (size_t)PB * W1;                      // PB * PB
    T* bsl = LD + PB * PB;                                // Wn
    T* yP = bsl + Wn;                                     // PB
    T* LDi = yP + PB;                                     // PB reciprocal pivots
    double* fakw = reinterpret_cast<double*>(LDi + PB);   // Wn
    double* fakN = fakw + Wn;                             // PB
    unsigned short* tXY = reinterpret_cast<unsigned short*>(fakN + PB);   // NTT
    unsigned char* dfw = reinterpret_cast<unsigned char*>(tXY + NTT);     // Wn: Dirichlet flag per slot
    __shared__ unsigned char dfN[PB];                                     // flags of the staged rows
    __shared__ T colb[32];                                                // column broadcast of the block factor
    __shared__ int s_err;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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

    for (int i = tid; i < NTT * TSTRIDE; i += NT) win[i] = Sc<T>::zero();
    for (int i = tid; i < PB * W1; i += NT) stage[i] = Sc<T>::zero();
    for (int i = tid; i < Wn; i += NT) {
        bsl[i] = Sc<T>::zero();
        fakw[i] = 0.0;
        dfw[i] = 0;
    }
    for (int t = tid; t < NTT; t += NT) {
        // decode t -> (X, Y) with X >= Y
        int X = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (tile_base(X + 1, 0) <= t) ++X;
        while (tile_base(X, 0) > t) --X;
        tXY[t] = (unsigned short)((X << 8) | (t - tile_base(X, 0)));
    }
    if (tid == 0) s_err = 0;
    __syncthreads();

    // Raw entries of rows [r0, r0 + PB) into stage[q][d].  The entries of
    // consecutive rows are contiguous in the gather lists, so the threads in
    // [t0, NT) take one entry each across all PB rows.
    auto stage_rows = [&](int r0, int t0) {
        if (r0 >= n) return;
        const int rend = min(r0 + PB, n);
        const int e0 = A.row_ptr[r0], e1 = A.row_ptr[rend];
        for (int e = e0 + (tid - t0); e < e1; e += NT - t0) {
            int q = 0;
            while (q + 1 < rend - r0 && A.row_ptr[r0 + q + 1] <= e) ++q;
            stage[q * W1 + A.ent_d[e]] = assemble_entry_b(A, e, k, l);
        }
    };
    // Scaling factors of the staged rows (threads q < PB).
    auto stage_fak = [&](int r0) {
        if (tid < PB) {
            const int r = r0 + tid;
            double f = 1.0;
            const unsigned char fl = (r < n) ? A.dflag[r] : 0;
            dfN[tid] = fl;
            if (r < n) {
                T raw = fl ? Sc<T>::one() : stage[tid * W1];
                double d = Sc<T>::absval(raw);
                if (!(d > 0.0)) s_err = CRT_ERR_ZERO_DIAG;
                else f = 1.0 / sqrt(d);
                fk[r] = f;
            }
            fakN[tid] = f;
        }
    };
    // Scaled staged rows into slots s_new .. s_new+PB-1; the window after the
    // write holds rows [wlo, wlo + Wn).  Every pair of a new slot with a row
    // c <= r is written (zero outside the band), pairs with later new rows
    // are written by those rows.
    auto scatter_rows = [&](int r0, int s_new, int wlo) {
        const int wm = wlo % Wn;
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const int r = r0 + q;
            const bool dr = dfN[q] != 0;
            for (int y = tid; y < Wn; y += NT) {
                int off = y - wm;
                if (off < 0) off += Wn;
                const int c = wlo + off;                      // row held by slot y
                if (c > r) continue;
                const int d = r - c;
                T v = Sc<T>::zero();
                if (r < n) {
                    if (d == 0) {
                        T raw = dr ? Sc<T>::one() : stage[q * W1];
                        v = Sc<T>::normalise(raw, Sc<T>::absval(raw));
                    } else if (d <= mb) {
                        const bool newc = c >= r0;
                        const bool dc = newc ? (dfN[c - r0] != 0) : (dfw[y] != 0);
                        if (!dr && !dc) {
                            const double fc = newc ? fakN[c - r0] : fakw[y];
                            v = scale(stage[q * W1 + d], fakN[q] * fc);
                        }
                    }
                }
                win[widx(s_new + q, y)] = v;
            }
        }
        __syncthreads();
        if (tid < PB) {
            const int r = r0 + tid;
            fakw[s_new + tid] = fakN[tid];
            dfw[s_new + tid] = dfN[tid];
            T bb = Sc<T>::zero();
            if (fuse && r < n) bb = scale(rhs_entry_b<T>(r, src, A.lsink, A.nsink0, A.dflag, A.dval, bdir), fakN[tid]);
            bsl[s_new + tid] = bb;
        }
        for (int i = tid; i < PB * W1; i += NT) stage[i] = Sc<T>::zero();
    };

    // Initial window: rows 0 .. Wn-1, PB at a time.
    for (int r0 = 0; r0 < Wn; r0 += PB) {
        stage_rows(r0, 0);
        __syncthreads();
        stage_fak(r0);
        __syncthreads();
        scatter_rows(r0, r0, 0);
        __syncthreads();
    }

    for (int i0 = 0; i0 < n; i0 += PB) {
        const int s0 = i0 % Wn;
        const int np_ = min(PB, n - i0);
        const int rnew0 = i0 + Wn;
        // ---- phase 1: diagonal block (warp 0) | next rows (warps 1..)
        if (warp == 0) {
            // lane j holds row j of the diagonal block; column t is broadcast
            // through colb[] (shared) once it is final
            T a[PB];
            T bj = Sc<T>::zero();
            const int j = lane;
            if (j < np_) {
#pragma unroll
                for (int t = 0; t < PB; ++t) a[t] = (t <= j && t < np_) ? win[widx(s0 + j, s0 + t)] : Sc<T>::zero();
                if (fuse) bj = bsl[s0 + j];
            } else {
#pragma unroll
                for (int t = 0; t < PB; ++t) a[t] = Sc<T>::zero();
            }
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                if (t >= np_) break;
                if (j == t) {
                    const T piv = a[t];
                    if (Sc<T>::bad_pivot(piv)) s_err = CRT_ERR_PIVOT;
                    const T ltt = Sc<T>::sqrt_fast(piv);
                    const T inv = Sc<T>::recip(ltt);
                    a[t] = ltt;
                    LDi[t] = inv;
                    if (fuse) {
                        bj = Sc<T>::mul(bj, inv);
                        yP[t] = bj;
                    }
                }
                __syncwarp();
                const T inv = LDi[t];
                if (j > t && j < np_) {
                    a[t] = Sc<T>::mul(a[t], inv);
                    colb[j] = a[t];
                }
                __syncwarp();
                // rank-1 update of the remaining block columns and the RHS
#pragma unroll
                for (int t2 = t + 1; t2 < PB; ++t2)
                    if (j >= t2 && j < np_) a[t2] -= Sc<T>::mul(a[t], colb[t2]);
                if (fuse && j > t && j < np_) bj -= Sc<T>::mul(a[t], yP[t]);
                __syncwarp();
            }
            if (j < np_) {
#pragma unroll
                for (int t = 0; t < PB; ++t) {
                    if (t <= j) {
                        LD[j * PB + t] = a[t];
                        if (j - t <= mb) Lc[(size_t)(i0 + t) * W1 + (j - t)] = a[t];
                    }
                }
                if (fuse) yv[i0 + j] = yP[j];
            }
        } else {
            stage_rows(rnew0, 32);
        }
        __syncthreads();
        // PROBE0
        if (s_err) break;
        // ---- phase 2: rows below the panel solve against the block
        stage_fak(rnew0);
        for (int x = tid; x < Wn; x += NT) {
            int dx = x - s0;
            if (dx < 0) dx += Wn;
            if (dx < PB) continue;                         // panel slot
            const int r = i0 + dx;
            if (r >= n || dx > mb + PB - 1) continue;
            T lx[PB];
#pragma unroll
            for (int t = 0; t < PB; ++t) lx[t] = (t < np_) ? win[widx(x, s0 + t)] : Sc<T>::zero();
            T bx = fuse ? bsl[x] : Sc<T>::zero();
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                if (t >= np_) break;
                T s = lx[t];
#pragma unroll
                for (int t2 = 0; t2 < t; ++t2) s -= Sc<T>::mul(lx[t2], LD[t * PB + t2]);
                lx[t] = Sc<T>::mul(s, LDi[t]);
                if (fuse) bx -= Sc<T>::mul(lx[t], yP[t]);
                win[widx(x, s0 + t)] = lx[t];
                const int d = r - (i0 + t);
                if (d <= mb) Lc[(size_t)(i0 + t) * W1 + d] = lx[t];
            }
            if (fuse) bsl[x] = bx;
        }
        __syncthreads();
        // PROBE1
        // ---- phase 3: trailing update T_xy -= L_x L_y^T on 4 x 4 tiles
        {
            const int P0 = s0 >> 2, P1 = (s0 + PB) >> 2;   // panel tile rows [P0, P1)
            for (int tt = tid; tt < NTT; tt += NT) {
                const int X = tXY[tt] >> 8, Y = tXY[tt] & 0xff;
                if ((X >= P0 && X < P1) || (Y >= P0 && Y < P1)) continue;
                T acc[16];
                T* tp = win + tt * TSTRIDE;
#pragma unroll
                for (int q = 0; q < 16; ++q) acc[q] = tp[q];
                for (int t = 0; t < np_; ++t) {
                    T px[4], py[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) px[a] = win[widx(4 * X + a, s0 + t)];
                    if (X == Y) {
#pragma unroll
                        for (int a = 0; a < 4; ++a) py[a] = px[a];
                    } else {
#pragma unroll
                        for (int a = 0; a < 4; ++a) py[a] = win[widx(4 * Y + a, s0 + t)];
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < 4; ++c) acc[a * 4 + c] -= Sc<T>::mul(px[a], py[c]);
                }
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    if (X == Y && (q >> 2) < (q & 3)) continue;   // upper half of a diagonal tile is unused
                    tp[q] = acc[q];
                }
            }
        }
        __syncthreads();
        // PROBE2
        // ---- phase 4: the staged rows enter the freed panel slots
        scatter_rows(rnew0, s0, i0 + PB);
        __syncthreads();
        // PROBE3
    }
    if (tid == 0) A.status[sys] = s_err;
}

}  // namespace

template <typename T, int PB>
static size_t blk_smem(int mb, int* Wn_out)
{
    const int Wn = ((mb + PB + PB - 1) / PB) * PB;
    const int NTR = Wn / 4, NTT = NTR * (NTR + 1) / 2;
    size_t s = (size_t)NTT * TSTRIDE * sizeof(T) + (size_t)PB * (mb + 1) * sizeof(T) + (size_t)PB * PB * sizeof(T) +
               (size_t)Wn * sizeof(T) + 2 * PB * sizeof(T) + (size_t)Wn * 8 + PB * 8 + (size_t)NTT * 2 + Wn + 64;
    *Wn_out = Wn;
    return s;
}

template <typename T>
bool launch_band_factor_blk(const BandArgs<T>& a, cudaStream_t st)
{
    constexpr int NT = 256, PB = 8;
    int Wn = 0;
    const size_t smem = blk_smem<T, PB>(a.mb, &Wn);
    if (smem > 227 * 1024 || Wn / 4 > 255) return false;
    cudaFuncSetAttribute(k_band_factor_blk<T, PB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_band_factor_blk<T, PB, NT><<<a.nsys, NT, smem, st>>>(a, Wn);
    return true;
}

template bool launch_band_factor_blk<double>(const BandArgs<double>&, cudaStream_t);
template bool launch_band_factor_blk<cd>(const BandArgs<cd>&, cudaStream_t);
