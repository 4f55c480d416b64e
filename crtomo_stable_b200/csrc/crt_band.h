// crt_band.h -- batched band factorisation and solves (kompab/kompadc +
// randb + scalab/scaldc + chol/choldc + vre/vredc in one streamed pass).
#pragma once

#include "crt_common.cuh"

template <typename T>
struct BandArgs {
    int n, mb, W;            // W = mb + 1 window slots
    int sys0, nsys;          // systems of this launch: sys0 .. sys0+nsys-1
    int L, K;                // electrodes, wavenumbers
    int mixed;               // 1: system s is (k = s / L, l = s % L) with its own matrix
    int fuse_rhs;            // 1: forward-substitute the system's own RHS in the factor pass
    int E, R, nmn;
    // gather lists (AssemblyLists, device copies)
    const int *row_ptr, *ent_d, *ent_ptr, *con_code, *con_sig;
    const double *elbg, *relbg, *kg;   // [K][E][nmn], [R][3], [K][L][R]
    const cd* sigma;                   // [E]
    const unsigned char* dflag;        // [n] 0 free, 1 type-13 node, 2 boundary.dat node
    const cd* dval;                    // [n] boundary.dat values (for dflag == 2)
    const cd* bdir;                    // [nsys][n] RHS moves of boundary.dat values, or NULL
    const int* enr0;                   // [L] 0-based electrode nodes
    int lsink, nsink0;
    // workspaces, indexed by b = blockIdx.x (system sys0 + b)
    T* Lws;                  // column-packed factor: column c at Lws[b*lstride + c*W + d], d = row - c
    size_t lstride;
    T* yws;                  // [b][n] forward-substitution result
    double* fakws;           // [b][n] scaling factors
    int* status;             // [total systems] errnr per system
    cd* aval;                // [b][row_ptr[n]] the prepared (scaled, edited) entries in FP64, or NULL
    size_t aval_stride;
    // k_band_factor_blk publishes its progress for a concurrent consumer:
    // progress[b] = c once columns [0, c) of system b are final (n at the
    // end, also after a failure); started counts the CTAs that have begun
    int* progress = nullptr;
    int* started = nullptr;
};

// One assembled band entry of system (k, l): kompab's sum over the entry's
// element and mixed-boundary contributions (src/kompab.f90:80-128), formed in
// the arithmetic W (FP64 or complex128) from the gather lists of A.
template <typename W, typename T>
__device__ __forceinline__ W band_assemble_entry(const BandArgs<T>& A, int e, int k, int l)
{
    W v = Sc<W>::zero();
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
        v += scale(Sc<W>::from(A.sigma[A.con_sig[c]]), coef);
    }
    return v;
}

// The area (part 0) or mixed-boundary (part 1) contributions of one band
// entry: the boundary coefficients kg averaged over the electrodes l0 ..
// l0 + nl - 1 (nl = 1: electrode l0's).
template <typename W, typename T>
__device__ __forceinline__ W band_assemble_part(const BandArgs<T>& A, int e, int k, int l0, int nl, int part)
{
    W v = Sc<W>::zero();
    const int c1 = A.ent_ptr[e + 1];
    const double* elbg_k = A.elbg + (size_t)k * A.E * A.nmn;
    for (int c = A.ent_ptr[e]; c < c1; ++c) {
        const int code = A.con_code[c];
        double coef;
        if (code >= 0) {
            if (part != 0) continue;
            coef = elbg_k[code];
        } else {
            if (part != 1) continue;
            const int q = -code - 1;
            const double* kq = A.kg + ((size_t)k * A.L + l0) * A.R + q / 3;
            double sk = 0.0;
            for (int j = 0; j < nl; ++j) sk += kq[(size_t)j * A.R];
            coef = A.relbg[q] * (sk / nl);
        }
        v += scale(Sc<W>::from(A.sigma[A.con_sig[c]]), coef);
    }
    return v;
}

template <typename T>
struct SolveArgs {
    int n, mb, W;
    int sys0, nsys, L, mixed;
    int lsink, nsink0;
    const int* enr0;
    const T* Lws;            // factor per workspace slot
    size_t lstride;
    const double* fakws;     // [slot][n]
    const T* yws;            // [slot][n] for fused systems (else NULL)
    int factor_of_sys_div;   // workspace slot of system s: (s - sys0) / factor_of_sys_div
    cd* kpot;                // kpot(sanz, eanz, kwnanz) Fortran order
    int* status;
    const T* rhs;            // [b][n] explicit right-hand sides (refinement), or NULL
    int accumulate;          // 1: kpot += the solution's contribution instead of kpot =
    // refinement: system b is skipped once refine_done(skip_omega, b,
    // skip_tau); NULL solves every system
    const unsigned long long* skip_omega;
    double skip_tau;
};

// Normwise backward error of refinement system b from om[2b] = max_r |r_r|
// and om[2b + 1] = max_r (sum_c |a_rc| |z_c| + |b_r|) (bits of non-negative
// doubles, |x| = |Re x| + |Im x|): converged when the ratio is at most tau.
__device__ __forceinline__ bool refine_done(const unsigned long long* om, int b, double tau)
{
    const double r = __longlong_as_double((long long)om[2 * b]);
    const double d = __longlong_as_double((long long)om[2 * b + 1]);
    return r <= tau * d;
}

template <typename T> void launch_band_factor(const BandArgs<T>& a, cudaStream_t st);
// Launch configuration of the panel-blocked variant: the panel width (4, 8
// or 16) in the low bits, BAND_CFG_WIDE for one 512-thread CTA per SM where
// the window would also fit twice (two 256-thread CTAs otherwise),
// BAND_CFG_NARROW for four 128-thread CTAs per SM where it fits four times.
constexpr int BAND_PANEL_MASK = 0xff;
constexpr int BAND_CFG_WIDE = 0x100;
constexpr int BAND_CFG_NARROW = 0x200;
// Panel-blocked variant in configuration cfg; returns false when its window
// does not fit in shared memory.
template <typename T> bool launch_band_factor_blk(const BandArgs<T>& a, int cfg, cudaStream_t st);
// Configuration for a's element type and half-bandwidth: the autotuned value
// of this process; the first call per (type, mb) measures the candidates on
// up to two waves of a's systems when may_tune (it prepares and factors
// them, so the caller prepares them again), else returns panel 8.
template <typename T> int band_panel(const BandArgs<T>& a, bool may_tune, cudaStream_t st);
// Whether the panel-blocked window fits in shared memory for half-bandwidth mb.
template <typename T> bool band_blk_fits(int mb);
// Preparation pass of the panel-blocked factor: assembled, Dirichlet-edited
// and scaled rows written row-packed into a.Lws, scaling factors into a.fakws.
template <typename T> void launch_band_prep(const BandArgs<T>& a, cudaStream_t st);
// Right-hand-side moves of non-zero boundary.dat values (randb2 / randbdc2)
// for a's systems: bdir[b][rows[i]] = sum_q value(node[q]) a(ent[q]) over
// q in [ptr[i], ptr[i+1]); the other rows of bdir are left as they are.
template <typename T>
void launch_band_dir_rhs(const BandArgs<T>& a, int nrows, const int* rows, const int* ptr, const int* ent,
                         const int* node, cd* bdir, cudaStream_t st);
// FP64 residual b^ - A^ z of the scaled systems for a refinement step, z from
// kpot, A^ from the entries the preparation pass kept in a.aval; solve
// systems sys0 .. sys0+nsolve-1, factor slot b / div; stored as T.
// Also the two maxima of each system's normwise backward error (see
// refine_done) into om_cur[2b], om_cur[2b + 1] (atomic maxima over the rows;
// om_cur zeroed beforehand).  A system that refine_done(om_prev, b, tau)
// reports converged at an earlier step (om_prev NULL: none) is not
// recomputed and its maxima carry over into om_cur.
template <typename T>
void launch_band_residual(const BandArgs<T>& a, int sys0, int nsolve, int div, const int* up_ptr, const int* up_ent,
                          const int* up_row, const cd* kpot, T* rout, const unsigned long long* om_prev,
                          unsigned long long* om_cur, double tau, cudaStream_t st);
// scratch: one n-vector per launched system (may alias the fused y workspace).
template <typename T> void launch_band_solve_with_scratch(const SolveArgs<T>& a, T* scratch, cudaStream_t st);
template <typename T> size_t band_factor_smem(int W);
