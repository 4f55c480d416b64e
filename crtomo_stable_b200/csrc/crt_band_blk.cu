// crt_band_blk.cu -- panel-blocked band factorisation (the production
// variant of k_band_factor, same inputs, outputs and arithmetic contract).
//
// A preparation pass (k_band_prep_diag / k_band_prep_rows, all rows of all
// systems in parallel) assembles every row from the gather lists (kompab),
// applies the Dirichlet edits (randb) and the symmetric scaling (scalab) in
// FP64 and stores the finished row r row-packed at Lws[r W + d] = A(r, r-d).
// That is exactly the place of column r of the column-packed factor, which
// is written only after row r has entered the window, so the factor
// overwrites the prepared matrix in place.
//
// One CTA per band system.  The panel width PB (4, 8 or 16) is chosen per
// element type and half-bandwidth by a measuring autotuner (band_panel).
// The window holds Wn = roundup(mb + PB, PB) rows
// in shared memory; row r lives in slot r mod Wn and the symmetric entry of
// two rows is stored once, at the unordered slot pair, in 4 x 4 tiles
// (tile (X, Y), X >= Y, row-major inside the tile).  Per panel of PB
// columns [i0, i0 + PB):
//   2. every window row below the panel solves its PB entries against the
//      block factor (L_x = A_x L_D^-T), updates its right-hand side and
//      writes its L entries to a panel buffer (t-major) and to the
//      column-packed HBM factor;
//   3a. the entries of the next panel's diagonal tiles receive the panel's
//      rank-PB update (one entry per thread);
//   3b. warp 0 factors the next PB x PB diagonal block (unconjugated L L^T,
//      the recurrence of src/chol.f90:44-78 restricted to the block) and
//      forward-substitutes its right-hand side, while warps 1.. update the
//      rest of the trailing window by the rank-PB product L_x L_y^T (each
//      thread accumulating 4 x 4 tiles in registers, the panel columns read
//      from the panel buffer), while the next PB prepared rows arrive in a
//      staging buffer by one bulk copy (cp.async.bulk with an mbarrier);
//      once all of them are through (a barrier of warps 1.. only), they
//      write the staged rows into the slots the panel freed.
// The first diagonal block is factored before the loop, so the serial
// block factorisation overlaps the trailing update of the previous panel.
#include "crt_band.h"

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

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

// One assembled band entry, formed in the arithmetic W.
template <typename W, typename T>
__device__ __forceinline__ W assemble_entry_w(const BandArgs<T>& A, int e, int k, int l)
{
    return band_assemble_entry<W>(A, e, k, l);
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

// System of launch slot b: (k, l) for mixed boundaries, else (k, 0).
template <typename T>
__device__ __forceinline__ void sys_kl(const BandArgs<T>& A, int sys, int& k, int& l)
{
    if (A.mixed) {
        k = sys / A.L;
        l = sys % A.L;
    } else {
        k = sys;
        l = 0;
    }
}

// Diagonal of every row: the normalised diagonal entry (scalab: unit modulus
// in the complex case, 1 in the real one; randb: 1 for a Dirichlet node) and
// the scaling factor fak = 1 / sqrt(|a_rr|); errnr 27 on a zero diagonal.
template <typename T>
__global__ void k_band_prep_diag(BandArgs<T> A)
{
    using WT = typename Wide<T>::type;   // formed in FP64, stored as T
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = A.n;
    if (idx >= (long long)A.nsys * n) return;
    const int b = (int)(idx / n), r = (int)(idx % n), sys = A.sys0 + b;
    int k, l;
    sys_kl(A, sys, k, l);
    WT raw = Sc<WT>::zero();
    int e0 = -1;
    for (int e = A.row_ptr[r]; e < A.row_ptr[r + 1]; ++e)
        if (A.ent_d[e] == 0) {
            raw = assemble_entry_w<WT>(A, e, k, l);
            e0 = e;
        }
    if (A.dflag[r]) raw = Sc<WT>::one();
    const double d = Sc<WT>::absval(raw);
    double f = 1.0;
    if (!(d > 0.0)) A.status[sys] = CRT_ERR_ZERO_DIAG;
    else f = 1.0 / sqrt(d);
    A.fakws[(size_t)b * n + r] = f;
    const WT dn = Sc<WT>::normalise(raw, d);
    A.Lws[(size_t)b * A.lstride + (size_t)r * A.W] = narrow<T>(dn);
    if (A.aval && e0 >= 0) A.aval[(size_t)b * A.aval_stride + e0] = Sc<WT>::to_cd(dn);
}

// randb2 / randbdc2 (src/randb2.f90:39-79): the couplings of the prescribed
// boundary.dat values move to the right-hand side of the free rows before
// scaling, b(r) += value(c) a(r, c) for every boundary.dat node c coupled to
// row r, with a the assembled (unscaled, FP64) entry of the system.  One
// thread per (system, row with couplings); couplings listed per row
// (ptr / ent / node: the gather entry of a(max(r,c), |r-c|) and c).  The
// real path takes the real part of the values through Sc<double>::from.
template <typename T>
__global__ void k_band_dir_rhs(BandArgs<T> A, int nrows, const int* __restrict__ rows, const int* __restrict__ ptr,
                               const int* __restrict__ ent, const int* __restrict__ node, cd* __restrict__ bdir)
{
    using WT = typename Wide<T>::type;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)A.nsys * nrows) return;
    const int b = (int)(idx / nrows), i = (int)(idx % nrows), sys = A.sys0 + b;
    int k, l;
    sys_kl(A, sys, k, l);
    cd s{0.0, 0.0};
    for (int q = ptr[i]; q < ptr[i + 1]; ++q)
        s += Sc<WT>::to_cd(assemble_entry_w<WT>(A, ent[q], k, l)) * A.dval[node[q]];
    bdir[(size_t)b * A.n + rows[i]] = s;
}

// Off-diagonal entries of every row, PREP_G lanes per row (a row has a
// handful of entries below the diagonal, so a warp serves 32 / PREP_G rows):
// zero fill, then a(r, r-d) * fak_r * fak_(r-d), or 0 when either node is a
// Dirichlet node.
constexpr int PREP_G = 8;

template <typename T>
__global__ void k_band_prep_rows(BandArgs<T> A)
{
    const long long gid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / PREP_G;
    const int lane = threadIdx.x % PREP_G, n = A.n;
    // every lane reaches the warp barrier: the zero fill must be visible
    // before any lane of the row writes an entry
    const bool active = gid < (long long)A.nsys * n;
    const int b = active ? (int)(gid / n) : 0, r = active ? (int)(gid % n) : 0, sys = A.sys0 + b;
    T* row = A.Lws + (size_t)b * A.lstride + (size_t)r * A.W;
    if (active) {
        if constexpr (std::is_same<T, cf>::value) {
            // complex64 rows start on 16-byte boundaries (even column stride):
            // entry 1 alone, then pairs (2m, 2m+1) by 16-byte stores; the last
            // pair may touch entry mb + 1, the row's padding
            if (lane == 0) row[1] = Sc<T>::zero();
            float4* pairs = reinterpret_cast<float4*>(row);
            for (int m = 1 + lane; 2 * m <= A.mb; m += PREP_G) pairs[m] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            for (int d = 1 + lane; d <= A.mb; d += PREP_G) row[d] = Sc<T>::zero();
        }
    }
    __syncwarp();
    if (!active) return;
    int k, l;
    sys_kl(A, sys, k, l);
    const double* fk = A.fakws + (size_t)b * n;
    const bool dr = A.dflag[r] != 0;
    const double fr = fk[r];
    for (int e = A.row_ptr[r] + lane; e < A.row_ptr[r + 1]; e += PREP_G) {
        const int d = A.ent_d[e];
        if (d == 0) continue;
        const int c = r - d;
        typename Wide<T>::type v = Sc<typename Wide<T>::type>::zero();
        if (!dr && A.dflag[c] == 0) v = scale(assemble_entry_w<typename Wide<T>::type>(A, e, k, l), fr * fk[c]);
        row[d] = narrow<T>(v);
        if (A.aval) A.aval[(size_t)b * A.aval_stride + e] = Sc<typename Wide<T>::type>::to_cd(v);
    }
}

// Residual of the scaled system for one step of iterative refinement, in
// FP64:  r = b^ - A^ z  with  z_c = -kpot_c / fak_c  (kpot = -fak o z), A^
// the matrix the preparation pass formed (its FP64 entries kept per gather
// entry in A.aval: the scaled, Dirichlet-edited a(r, c) fak_r fak_c and the
// normalised diagonal), b^ = fak o rhs.  One thread per row of every
// system: the row's own entries give the lower part and the diagonal, the
// transposed list the upper part.  A Dirichlet row is the identity row.
// The residual is stored in T for the correction solve.  Solve system b is
// (k, l) = (sys0 + b) / L, % L, its factor slot b / div.
__device__ __forceinline__ double cabs1(cd v) { return fabs(v.x) + fabs(v.y); }

template <typename T>
__global__ void k_band_residual(BandArgs<T> A, int sys0, int nsolve, int div, const int* __restrict__ up_ptr,
                                const int* __restrict__ up_ent, const int* __restrict__ up_row,
                                const cd* __restrict__ kpot, T* rout, const unsigned long long* om_prev,
                                unsigned long long* om_cur, double tau)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = A.n;
    if (idx >= (long long)nsolve * n) return;
    const int b = (int)(idx / n), r = (int)(idx % n), sys = sys0 + b;
    if (om_prev && refine_done(om_prev, b, tau)) {   // converged at an earlier step
        if (r == 0) {
            om_cur[2 * b] = om_prev[2 * b];
            om_cur[2 * b + 1] = om_prev[2 * b + 1];
        }
        return;
    }
    const int l = sys % A.L, slot = b / div;
    const double* fk = A.fakws + (size_t)slot * n;
    const cd* kp = kpot + (size_t)sys * n;
    const cd* av = A.aval + (size_t)slot * A.aval_stride;
    auto zval = [&](int c) {
        const double inv = 1.0 / fk[c];   // one division for both components
        return cd{-kp[c].x * inv, -kp[c].y * inv};
    };
    cd acc{0.0, 0.0};
    double den = 0.0;   // sum_c |a_rc| |z_c|
    if (A.dflag[r]) {
        acc = zval(r);
        den = cabs1(acc);
    } else {
        for (int e = A.row_ptr[r]; e < A.row_ptr[r + 1]; ++e) {
            const cd a = av[e], zc = zval(r - A.ent_d[e]);
            acc += a * zc;
            den += cabs1(a) * cabs1(zc);
        }
        for (int q = up_ptr[r]; q < up_ptr[r + 1]; ++q) {
            const cd a = av[up_ent[q]], zc = zval(up_row[q]);
            acc += a * zc;
            den += cabs1(a) * cabs1(zc);
        }
    }
    // The refactored systems (every system with mixed boundaries, electrode
    // 1 otherwise) carry kompab's right-hand side with the Dirichlet edits
    // (randb / randb2, their boundary.dat couplings in bdir); the others are
    // kompb's (src/kompb.f90:39-66): -1 at the source, +1 at the sink, no
    // edits, as in the reference's loop.
    cd b0;
    if (A.mixed || l == 0) {
        const cd* bd = A.bdir ? A.bdir + (size_t)slot * n : nullptr;
        b0 = rhs_entry_b<cd>(r, A.enr0[l], A.lsink, A.nsink0, A.dflag, A.dval, bd);
    } else {
        b0 = cd{r == A.enr0[l] ? -1.0 : 0.0, 0.0};
        if (A.lsink && r == A.nsink0) b0 = cd{1.0, 0.0};
    }
    const cd bb = scale(b0, fk[r]);
    const cd res = bb - acc;
    rout[(size_t)b * n + r] = narrow<T>(res);
    if (om_cur) {
        // max |r_r| and max (sum_c |a_rc||z_c| + |b_r|) of the system: a warp
        // whose lanes all hold rows of one system reduces first (one atomic
        // per warp and quantity instead of one per row)
        unsigned long long vr = (unsigned long long)__double_as_longlong(cabs1(res));
        unsigned long long vd = (unsigned long long)__double_as_longlong(den + cabs1(bb));
        const unsigned mask = __activemask();
        const int lane = threadIdx.x & 31;
        const int b0 = __shfl_sync(mask, b, __ffs(mask) - 1);
        if (mask == 0xffffffffu && __all_sync(mask, b == b0)) {
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long ur = __shfl_xor_sync(mask, vr, o), ud = __shfl_xor_sync(mask, vd, o);
                vr = ur > vr ? ur : vr;
                vd = ud > vd ? ud : vd;
            }
            if (lane == 0) {
                atomicMax(&om_cur[2 * b], vr);
                atomicMax(&om_cur[2 * b + 1], vd);
            }
        } else {
            atomicMax(&om_cur[2 * b], vr);
            atomicMax(&om_cur[2 * b + 1], vd);
        }
    }
}

// Four consecutive window-row entries of a panel column (16-byte aligned).
template <typename T>
__device__ __forceinline__ void load4(const T* p, T (&v)[4])
{
#pragma unroll
    for (int a = 0; a < 4; ++a) v[a] = p[a];
}
template <>
__device__ __forceinline__ void load4<cf>(const cf* p, cf (&v)[4])
{
    const float4 u = *reinterpret_cast<const float4*>(p);
    const float4 w = *reinterpret_cast<const float4*>(p + 2);
    v[0] = cf{u.x, u.y};
    v[1] = cf{u.z, u.w};
    v[2] = cf{w.x, w.y};
    v[3] = cf{w.z, w.w};
}

// Panel buffer padding (see the kernel): complex64 reads four entries with
// two 16-byte loads and keeps the rows unpadded (16-byte aligned).
template <typename T> struct PanPad { static constexpr bool v = true; };
template <> struct PanPad<cf> { static constexpr bool v = false; };

// Staged rows copied by one bulk copy (16-byte aligned, a multiple of 16
// bytes): complex entries (8 or 16 bytes, and the complex64 column stride is
// even), so every row run starts on a 16-byte boundary; real FP64 rows may
// not.
template <typename T> struct StageAsync { static constexpr bool v = true; };
template <> struct StageAsync<double> { static constexpr bool v = false; };

template <typename T, int PB, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_band_factor_blk(BandArgs<T> A, int Wn)
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
    double* fakN = reinterpret_cast<double*>(LDi + PB);   // PB scaling factors of the staged rows
    unsigned short* tXY = reinterpret_cast<unsigned short*>(fakN + PB);   // NTT tile coordinates
    // the panel's columns L(x, i0 + t) of every window row x, t-major
    // (pan[t Wn + x]): the trailing updates read them here, so the panel's
    // slots of the window are free for the next rows while they run
    T* pan = reinterpret_cast<T*>((reinterpret_cast<size_t>(tXY + NTT) + 15) & ~(size_t)15);
    // row x of a panel column at ppos(x); entry types without the 16-byte
    // vector loads pad every tile row of 4 by one entry, so the tile rows a
    // warp reads at once fall into different banks
    constexpr bool PAN_PAD = PanPad<T>::v;
    const int PS = PAN_PAD ? Wn + Wn / 4 : Wn;   // stride between panel columns
    auto ppos = [&](int x) { return PAN_PAD ? x + (x >> 2) : x; };
    __shared__ T colb[32];                                                // column broadcast of the block factor
    __shared__ T bN[PB];                                                  // scaled right-hand side of the staged rows
    __shared__ int s_err;
    __shared__ __align__(8) unsigned long long s_bar;   // mbarrier of the staged rows' bulk copy

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x, sys = A.sys0 + b;
    // progress for a consumer that sweeps the finished columns while this
    // CTA goes on: published by the last thread after a barrier
    auto publish = [&](int c) {
        if (A.progress && tid == NT - 1) {
            __threadfence();
            asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(A.progress + b), "r"(c) : "memory");
        }
    };
    if (A.started && tid == 0) atomicAdd(A.started, 1);
    if (A.status[sys] != 0) {   // zero diagonal found by the preparation pass
        publish(A.n);
        return;
    }
    int k, l;
    sys_kl(A, sys, k, l);
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
    }
    for (int t = tid; t < NTT; t += NT) {
        // decode t -> (X, Y) with X >= Y
        int X = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (tile_base(X + 1, 0) <= t) ++X;
        while (tile_base(X, 0) > t) --X;
        tXY[t] = (unsigned short)((X << 8) | (t - tile_base(X, 0)));
    }
    if (tid == 0) {
        s_err = 0;
        mbar_init(&s_bar, 1);
    }
    int bar_phase = 0;
    __syncthreads();

    // Prepared rows [r0, r0 + PB) into stage[q][d] and their scaling factors
    // into fakN (threads t0 .. NT-1; rows beyond n are zero).
    // per-row scaling factors and right-hand sides of the staged rows
    auto row_meta = [&](int r0, int t0) {
        const int q = tid - t0;
        if (q >= 0 && q < PB) {
            const int r = r0 + q;
            const double f = (r < n) ? fk[r] : 1.0;
            fakN[q] = f;
            T bb = Sc<T>::zero();
            if (fuse && r < n) bb = scale(rhs_entry_b<T>(r, src, A.lsink, A.nsink0, A.dflag, A.dval, bdir), f);
            bN[q] = bb;
        }
    };
    auto load_rows = [&](int r0, int t0) {
        const T* src_rows = Lc + (size_t)r0 * W1;
        for (int i = tid - t0; i < PB * W1; i += NT - t0) {
            const int q = i / W1;
            stage[i] = (r0 + q < n) ? src_rows[i] : Sc<T>::zero();
        }
        row_meta(r0, t0);
    };
    // Staged rows into slots s_new .. s_new+PB-1; the window after the write
    // holds rows [wlo, wlo + Wn).  Every pair of a new slot with a row
    // c <= r is written (zero outside the band), pairs with later new rows
    // are written by those rows.
    auto scatter_rows = [&](int r0, int s_new, int wlo, int t0) {
        const int wm = wlo % Wn;
        for (int i = tid - t0; i < PB * Wn; i += NT - t0) {
            const int q = i % PB, y = i / PB;             // PB is a power of two
            int off = y - wm;
            if (off < 0) off += Wn;
            const int c = wlo + off;                      // row held by slot y
            const int r = r0 + q;
            if (c > r) continue;
            const int d = r - c;
            win[widx(s_new + q, y)] = (r < n && d <= mb) ? stage[q * W1 + d] : Sc<T>::zero();
        }
        if (tid - t0 >= 0 && tid - t0 < PB) bsl[s_new + tid - t0] = bN[tid - t0];
    };

    // Initial window: rows 0 .. Wn-1, PB at a time.
    for (int r0 = 0; r0 < Wn; r0 += PB) {
        load_rows(r0, 0);
        __syncthreads();
        scatter_rows(r0, r0, 0, 0);
        __syncthreads();
    }

    // Diagonal block of the panel starting at row p0 (warp 0): lane j holds
    // row j of the block; column t is broadcast through colb[] (shared)
    // once it is final.  Writes LD, the reciprocal pivots LDi, the panel's
    // forward-substituted RHS yP and the block's L entries.
    auto diag_block = [&](int p0) {
        const int sp = p0 % Wn, npp = min(PB, n - p0);
        T a[PB];
        T bj = Sc<T>::zero();
        const int j = lane;
        if (j < npp) {
#pragma unroll
            for (int t = 0; t < PB; ++t) a[t] = (t <= j && t < npp) ? win[widx(sp + j, sp + t)] : Sc<T>::zero();
            if (fuse) bj = bsl[sp + j];
        } else {
#pragma unroll
            for (int t = 0; t < PB; ++t) a[t] = Sc<T>::zero();
        }
#pragma unroll
        for (int t = 0; t < PB; ++t) {
            if (t >= npp) break;
            if (j == t) {
                const T piv = a[t];
                if (Sc<T>::bad_pivot(piv)) s_err = CRT_ERR_PIVOT;
                T ltt, inv;
                Sc<T>::sqrt_recip(piv, ltt, inv);
                a[t] = ltt;
                LDi[t] = inv;
                if (fuse) {
                    bj = Sc<T>::mul(bj, inv);
                    yP[t] = bj;
                }
            }
            __syncwarp();
            const T inv = LDi[t];
            if (j > t && j < npp) {
                a[t] = Sc<T>::mul(a[t], inv);
                colb[j] = a[t];
            }
            __syncwarp();
            // rank-1 update of the remaining block columns and the RHS
#pragma unroll
            for (int t2 = t + 1; t2 < PB; ++t2)
                if (j >= t2 && j < npp) fms_acc(a[t2], a[t], colb[t2]);
            if (fuse && j > t && j < npp) fms_acc(bj, a[t], yP[t]);
            __syncwarp();
        }
        if (j < npp) {
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                if (t <= j) {
                    LD[j * PB + t] = a[t];
                    if (j - t <= mb) Lc[(size_t)(p0 + t) * W1 + (j - t)] = a[t];
                }
            }
            if (fuse) yv[p0 + j] = yP[j];
        }
    };
    // the panel occupies tile rows [P0, P0 + NPT) of the window
    constexpr int NPT = PB / 4;

    if (warp == 0) diag_block(0);
    // the staging buffer's next writer is the async (bulk copy) proxy
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    for (int i0 = 0; i0 < n; i0 += PB) {
        if (s_err) break;
        const int s0 = i0 % Wn;
        const int np_ = min(PB, n - i0);
        const int rnew0 = i0 + Wn;
        const int P0 = s0 >> 2;
        // ---- phase 2: rows below the panel solve against the block
        for (int x = tid; x < Wn; x += NT) {
            int dx = x - s0;
            if (dx < 0) dx += Wn;
            if (dx < PB) continue;                         // panel slot
            const int r = i0 + dx;
            if (r >= n || dx > mb + PB - 1) {
#pragma unroll
                for (int t = 0; t < PB; ++t) pan[t * PS + ppos(x)] = Sc<T>::zero();
                continue;
            }
            T lx[PB];
#pragma unroll
            for (int p = 0; p < NPT; ++p) {
                // the row's entries of panel tile row P0 + p: tile (X, P) after the
                // panel in slot order (entry (x & 3, t & 3)), (P, X) before it
                const int X = x >> 2, P = P0 + p;
                const int base = (X > P ? tile_base(X, P) * TSTRIDE + ((x & 3) << 2)
                                        : tile_base(P, X) * TSTRIDE + (x & 3));
                const int step = X > P ? 1 : 4;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int t = 4 * p + u;
                    lx[t] = (t < np_) ? win[base + u * step] : Sc<T>::zero();
                }
            }
            T bx = fuse ? bsl[x] : Sc<T>::zero();
#pragma unroll
            for (int t = 0; t < PB; ++t) {
                if (t >= np_) {
                    pan[t * PS + ppos(x)] = Sc<T>::zero();
                    continue;
                }
                T s = lx[t];
#pragma unroll
                for (int t2 = 0; t2 < t; ++t2) fms_acc(s, lx[t2], LD[t * PB + t2]);
                lx[t] = Sc<T>::mul(s, LDi[t]);
                if (fuse) fms_acc(bx, lx[t], yP[t]);
                pan[t * PS + ppos(x)] = lx[t];
                const int d = r - (i0 + t);
                if (d <= mb) Lc[(size_t)(i0 + t) * W1 + d] = lx[t];
            }
            if (fuse) bsl[x] = bx;
        }
        __syncthreads();
        // columns [0, i0 + PB) are final (the diagonal blocks were written
        // by earlier phases); published every 16 panels
        if (((i0 / PB) & 15) == 15) publish(i0 + PB);
        // ---- phase 3a: the trailing update of the next panel's diagonal
        // tiles, one entry per thread, so that its block can be factored
        // while the rest of the window is updated.
        const int inext = i0 + PB;
        const bool has_next = inext < n;
        const int P0n = (inext % Wn) >> 2;
        if (has_next) {
            constexpr int NDT = NPT * (NPT + 1) / 2;
            for (int i = tid; i < NDT * 16; i += NT) {
                const int kt = i >> 4, q = i & 15;
                int xo = 0;
                while ((xo + 1) * (xo + 2) / 2 <= kt) ++xo;
                const int yo = kt - xo * (xo + 1) / 2;
                const int X = P0n + xo, Y = P0n + yo, a = q >> 2, c = q & 3;
                if (X == Y && a < c) continue;
                T* tp = win + tile_base(X, Y) * TSTRIDE + q;
                T acc = *tp;
#pragma unroll
                for (int t = 0; t < PB; ++t) {
                    if (t >= np_) break;
                    fms_acc(acc, pan[t * PS + ppos(4 * X) + a], pan[t * PS + ppos(4 * Y) + c]);
                }
                *tp = acc;
            }
        }
        __syncthreads();
        // ---- phase 3b: warp 0 factors the next diagonal block; warps 1..
        // update the rest of the window by the rank-PB product L_x L_y^T on
        // 4 x 4 tiles (the panel columns read from pan) and then write the
        // staged rows into the panel's slots.
        if (warp == 0) {
            if (has_next) diag_block(inext);
        } else {
            // the next PB prepared rows start their way into the staging
            // buffer (bulk copy) and arrive while the tiles are updated
            const char* srcb = reinterpret_cast<const char*>(Lc + (size_t)rnew0 * W1);
            char* dstb = reinterpret_cast<char*>(stage);
            const int bytes = PB * W1 * (int)sizeof(T);
            const bool async_rows = StageAsync<T>::v && rnew0 + PB <= n && (reinterpret_cast<size_t>(srcb) & 15) == 0 &&
                                    (reinterpret_cast<size_t>(dstb) & 15) == 0 && (bytes & 15) == 0;
            if (async_rows && tid == 32) {
                // one bulk copy (the TMA engine) of the PB contiguous rows
                mbar_expect_tx(&s_bar, bytes);
                bulk_g2s(dstb, srcb, bytes, &s_bar);
            }
            if (has_next) {
                for (int tt = tid - 32; tt < NTT; tt += NT - 32) {
                    const int X = tXY[tt] >> 8, Y = tXY[tt] & 0xff;
                    if ((X >= P0 && X < P0 + NPT) || (Y >= P0 && Y < P0 + NPT)) continue;
                    if (X >= P0n && X < P0n + NPT && Y >= P0n && Y < P0n + NPT) continue;   // done in 3a
                    T acc[16];
                    T* tp = win + tt * TSTRIDE;
#pragma unroll
                    for (int q = 0; q < 16; ++q) acc[q] = tp[q];
#pragma unroll
                    for (int t = 0; t < PB; ++t) {
                        if (t >= np_) break;
                        T px[4], py[4];
                        load4(pan + t * PS + ppos(4 * X), px);
                        load4(pan + t * PS + ppos(4 * Y), py);
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int c = 0; c < 4; ++c) fms_acc(acc[a * 4 + c], px[a], py[c]);
                    }
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        if (X == Y && (q >> 2) < (q & 3)) continue;   // upper half of a diagonal tile is unused
                        tp[q] = acc[q];
                    }
                }
            }
            if (async_rows) {
                if (!mbar_wait(&s_bar, bar_phase)) s_err = CRT_ERR_CUDA;
                bar_phase ^= 1;
                row_meta(rnew0, 32);
            } else {
                load_rows(rnew0, 32);
            }
            // warps 1.. only (warp 0 is in the diagonal block): the staged rows
            // are visible, and every tile update is done, so the panel's
            // slots take the new rows
            asm volatile("bar.sync 1, %0;\n" ::"r"(NT - 32) : "memory");
            scatter_rows(rnew0, s0, i0 + PB, 32);
            // the staging buffer's next writer is the async (bulk copy) proxy
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        }
        __syncthreads();
    }
    if (tid == 0 && s_err) A.status[sys] = s_err;
    publish(n);
}

}  // namespace

template <typename T, int PB>
static size_t blk_smem(int mb, int* Wn_out)
{
    const int Wn = ((mb + PB + PB - 1) / PB) * PB;
    const int NTR = Wn / 4, NTT = NTR * (NTR + 1) / 2;
    size_t s = (size_t)NTT * TSTRIDE * sizeof(T) + (size_t)PB * (mb + 1) * sizeof(T) + (size_t)PB * PB * sizeof(T) +
               (size_t)Wn * sizeof(T) + 2 * PB * sizeof(T) + (size_t)Wn * 8 + PB * 8 + (size_t)NTT * 2 + Wn + 64 +
               (size_t)PB * (Wn + Wn / 4) * sizeof(T) + 16;
    *Wn_out = Wn;
    return s;
}

template <typename T>
static size_t blk_smem_pb(int pb, int mb, int* Wn)
{
    switch (pb) {
    case 4: return blk_smem<T, 4>(mb, Wn);
    case 16: return blk_smem<T, 16>(mb, Wn);
    default: return blk_smem<T, 8>(mb, Wn);
    }
}

template <typename T>
static bool blk_fits_pb(int pb, int mb)
{
    int Wn = 0;
    const size_t smem = blk_smem_pb<T>(pb, mb, &Wn);
    return smem <= 227 * 1024 && Wn / 4 <= 255;
}

template <typename T>
bool band_blk_fits(int mb)
{
    return blk_fits_pb<T>(8, mb);
}

template <typename T>
void launch_band_prep(const BandArgs<T>& a, cudaStream_t st)
{
    const long long rows = (long long)a.nsys * a.n;
    k_band_prep_diag<T><<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(a);
    k_band_prep_rows<T><<<(unsigned)((rows * PREP_G + 255) / 256), 256, 0, st>>>(a);
}

template <typename T>
void launch_band_dir_rhs(const BandArgs<T>& a, int nrows, const int* rows, const int* ptr, const int* ent,
                         const int* node, cd* bdir, cudaStream_t st)
{
    const long long m = (long long)a.nsys * nrows;
    if (m > 0) k_band_dir_rhs<T><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(a, nrows, rows, ptr, ent, node, bdir);
}

// Threads per CTA of a launch configuration for a window of smem bytes: a
// window that fits twice per SM runs as two 256-thread CTAs (one system's
// serial phases overlap the other's update), a small one may run as four
// 128-thread CTAs (BAND_CFG_NARROW), a large one (or BAND_CFG_WIDE) as one
// CTA of 512.  0: the configuration does not fit.
static int cfg_threads(int cfg, size_t smem)
{
    constexpr size_t lim = 227 * 1024;
    if (cfg & BAND_CFG_NARROW) return 4 * smem <= lim ? 128 : 0;
    if (!(cfg & BAND_CFG_WIDE) && 2 * smem <= lim) return 256;
    return smem <= lim ? 512 : 0;
}

template <typename T, int PB>
static void launch_blk_pb(const BandArgs<T>& a, int cfg, cudaStream_t st)
{
    int Wn = 0;
    const size_t smem = blk_smem<T, PB>(a.mb, &Wn);
    auto go = [&](auto kern, int nt) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<a.nsys, nt, smem, st>>>(a, Wn);
    };
    switch (cfg_threads(cfg, smem)) {
    case 128: go(k_band_factor_blk<T, PB, 128, 4>, 128); break;
    case 256: go(k_band_factor_blk<T, PB, 256, 2>, 256); break;
    default: go(k_band_factor_blk<T, PB, 512, 1>, 512); break;
    }
}

template <typename T>
bool launch_band_factor_blk(const BandArgs<T>& a, int cfg, cudaStream_t st)
{
    const int pb = cfg & BAND_PANEL_MASK;
    if (!blk_fits_pb<T>(pb, a.mb)) return false;
    int Wn = 0;
    if (cfg_threads(cfg, blk_smem_pb<T>(pb, a.mb, &Wn)) == 0) cfg = pb;
    switch (pb) {
    case 4: launch_blk_pb<T, 4>(a, cfg, st); break;
    case 16: launch_blk_pb<T, 16>(a, cfg, st); break;
    default: launch_blk_pb<T, 8>(a, cfg, st); break;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Panel-width autotuner.  The best panel (4, 8 or 16 columns) and CTA shape
// (two 256-thread CTAs per SM where the window fits twice, four of 128 where
// it fits four times, or one of 512)
// depend on the element type and the half-bandwidth (window size, CTAs per
// SM, serial panel phases against the rank-PB update); they are measured once per
// (type, mb) in the process on the first systems of a real chunk: for each
// candidate that fits, the preparation pass and the factorisation of up to
// two waves of systems are run and the factorisation is timed with events.
// The caller's real pass then prepares and factors the chunk again, so the
// trials leave no trace but their per-system status, which is cleared.
// CRT_B200_PANEL = 4 | 8 | 16 fixes the width (with CRT_B200_FACTOR_CTA =
// 128 | 256 | 512 the CTA shape where the window allows it);
// CRT_B200_TUNE_LOG prints the trials to stderr.
namespace {
std::mutex g_panel_mu;
std::map<std::pair<int, int>, int> g_panel;   // (sizeof(T), mb) -> launch configuration
}

template <typename T>
int band_panel(const BandArgs<T>& a, bool may_tune, cudaStream_t st)
{
    if (const char* env = std::getenv("CRT_B200_PANEL")) {
        const int pb = std::atoi(env);
        if ((pb == 4 || pb == 8 || pb == 16) && blk_fits_pb<T>(pb, a.mb)) {
            int cfg = pb;
            if (const char* ce = std::getenv("CRT_B200_FACTOR_CTA")) {
                const int nt = std::atoi(ce);
                cfg |= nt == 128 ? BAND_CFG_NARROW : nt == 512 ? BAND_CFG_WIDE : 0;
            }
            return cfg;
        }
    }
    int nsm = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // tuned separately for launches of at most one system per SM (the
    // interior systems of the Schur form: one per wavenumber), where no
    // second system shares an SM
    const int few = a.nsys <= nsm ? 1 : 0;
    const std::pair<int, int> key(((int)sizeof(T) << 1) | few, a.mb);
    {
        std::lock_guard<std::mutex> g(g_panel_mu);
        auto it = g_panel.find(key);
        if (it != g_panel.end()) return it->second;
    }
    if (!may_tune) return 8;
    BandArgs<T> t = a;
    t.nsys = std::min(a.nsys, 2 * nsm);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 8;
    float best_ms = 1e30f;
    for (int cfg : {8, 4, 16, 8 | BAND_CFG_WIDE, 4 | BAND_CFG_WIDE, 8 | BAND_CFG_NARROW, 4 | BAND_CFG_NARROW}) {
        const int pb = cfg & BAND_PANEL_MASK;
        if (!blk_fits_pb<T>(pb, a.mb)) continue;
        int Wn = 0;
        const size_t sm = blk_smem_pb<T>(pb, a.mb, &Wn);
        const int nt = cfg_threads(cfg, sm);
        if (nt == 0) continue;
        if ((cfg & BAND_CFG_WIDE) && cfg_threads(pb, sm) == 512) continue;   // the same as pb alone
        launch_band_prep<T>(t, st);
        cudaEventRecord(e0, st);
        launch_band_factor_blk<T>(t, cfg, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (std::getenv("CRT_B200_TUNE_LOG"))
            std::fprintf(stderr, "band factor autotune: %d-byte entries, mb %d, panel %d, %d threads: %.3f ms\n",
                         (int)sizeof(T), a.mb, pb, nt, ms);
        if (ms < best_ms) {
            best_ms = ms;
            best = cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemsetAsync(a.status + a.sys0, 0, sizeof(int) * (size_t)t.nsys, st);
    std::lock_guard<std::mutex> g(g_panel_mu);
    g_panel[key] = best;
    return best;
}

template <typename T>
void launch_band_residual(const BandArgs<T>& a, int sys0, int nsolve, int div, const int* up_ptr, const int* up_ent,
                          const int* up_row, const cd* kpot, T* rout, const unsigned long long* om_prev,
                          unsigned long long* om_cur, double tau, cudaStream_t st)
{
    const long long rows = (long long)nsolve * a.n;
    k_band_residual<T><<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(a, sys0, nsolve, div, up_ptr, up_ent, up_row,
                                                                     kpot, rout, om_prev, om_cur, tau);
}

template bool band_blk_fits<double>(int);
template bool band_blk_fits<cd>(int);
template bool band_blk_fits<cf>(int);
template void launch_band_dir_rhs<double>(const BandArgs<double>&, int, const int*, const int*, const int*,
                                          const int*, cd*, cudaStream_t);
template void launch_band_dir_rhs<cd>(const BandArgs<cd>&, int, const int*, const int*, const int*, const int*, cd*,
                                      cudaStream_t);
template void launch_band_dir_rhs<cf>(const BandArgs<cf>&, int, const int*, const int*, const int*, const int*, cd*,
                                      cudaStream_t);
template void launch_band_prep<double>(const BandArgs<double>&, cudaStream_t);
template void launch_band_prep<cd>(const BandArgs<cd>&, cudaStream_t);
template void launch_band_prep<cf>(const BandArgs<cf>&, cudaStream_t);
template bool launch_band_factor_blk<double>(const BandArgs<double>&, int, cudaStream_t);
template bool launch_band_factor_blk<cd>(const BandArgs<cd>&, int, cudaStream_t);
template bool launch_band_factor_blk<cf>(const BandArgs<cf>&, int, cudaStream_t);
template int band_panel<double>(const BandArgs<double>&, bool, cudaStream_t);
template int band_panel<cd>(const BandArgs<cd>&, bool, cudaStream_t);
template int band_panel<cf>(const BandArgs<cf>&, bool, cudaStream_t);
template void launch_band_residual<cf>(const BandArgs<cf>&, int, int, int, const int*, const int*, const int*,
                                       const cd*, cf*, const unsigned long long*, unsigned long long*, double,
                                       cudaStream_t);
