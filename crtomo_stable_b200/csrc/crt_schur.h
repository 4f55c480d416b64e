// crt_schur.h -- forward model by elimination of the mixed-boundary nodes.
//
// With mixed boundaries the reference assembles and factors one band system
// per wavenumber k and source electrode l (src/inv.f90:426-484,
// src/fem.f90:328-397): the electrode enters only through the boundary
// coefficients kg(rel, l, k) of the type-11 segments (src/kompab.f90:
// 113-117), which couple the nodes of those segments (the set G, m nodes)
// and nothing else.  Splitting the nodes into G and the interior I,
//
//     [ A_II   A_IG    ] [p_I]   [r_I]        A_II, A_IG independent of l,
//     [ A_GI   A_GG(l) ] [p_G] = [r_G]        r = e_src(l) - e_sink.
//
// With the interior factor F A_II F = L L^T (F = diag(fak), the scaled,
// unconjugated factorisation of the direct path), u^ = L^-1 F r_I and
// V^ = L^-1 F A_IG:
//
//     S_l p_G = r_G - V^T u^_l,     S_l = A_GG(l) - V^T V^,
//     p_I = F L^-T (u^_l - V^ p_G).
//
// Per wavenumber: one band factorisation of A_II, a forward sweep of the
// L + m columns [F r_I | F A_IG] (each from its first non-zero row) and the
// Gram products V^T [u^ | V^]; per (k, l) a dense m x m complex-symmetric
// Cholesky of S_l with its two triangular solves; then z^ = u^ - V^ p_G (a
// GEMM) and one back sweep per source column.  The arithmetic is FP64
// (complex128 or real) throughout; the result equals the reference's
// per-system elimination up to rounding (the same matrix, another
// elimination order).
#pragma once

#include <vector>

#include "crt_band.h"
#include "crt_setup.h"

// Largest boundary set the dense Schur kernels take (panel in shared memory).
constexpr int SCHUR_MMAX = 768;
// Columns per CTA of the forward sweep (all columns) and of the back sweep
// (the source columns), and the row block of both.
constexpr int SCHUR_MS_R = 32;
constexpr int SCHUR_BK_R = 16;
constexpr int SCHUR_MS_BB = 16;

// Host-side plan: node split, interior assembly lists, couplings.
struct SchurHost {
    int n = 0, nI = 0, m = 0, mbI = 0, L = 0;
    std::vector<int> permI;         // [nI] node of interior position i (ascending)
    std::vector<int> gam;           // [m] node of boundary position g (ascending)
    std::vector<int> posI_src;      // [L] interior position of electrode l's node, or -1
    std::vector<int> posG_src;      // [L] boundary position of electrode l's node, or -1
    int posI_sink = -1, posG_sink = -1;
    AssemblyLists lists_I;          // interior system A_II, rows = interior positions
    // G-I couplings, CSR by boundary position g: interior position and the
    // full mesh's gather entry of a(g-node, i-node)
    std::vector<int> gi_ptr, gi_pos, gi_ent, gi_g;
    // G-G entries (g >= h) of A_GG(l): full gather entries (area and
    // mixed-boundary contributions)
    std::vector<int> gg_g, gg_h, gg_ent;
    // rows of the mixed-boundary part D_l of A_GG(l) (both triangles): per
    // boundary position g, the columns h and gather entries of the G-G
    // entries with a mixed-boundary contribution
    std::vector<int> bd_ptr, bd_col, bd_ent;
    // multi-RHS solve: columns ordered by their first non-zero interior
    // row; blocks of SCHUR_MS_R columns and their first rows
    std::vector<int> col_order, blk_start;
    int R = SCHUR_MS_R;             // columns per block of the forward sweep (16 or 32)
    std::vector<int> first;         // [L + m] first non-zero interior row of each column
    std::vector<int> gsort, gfirst; // boundary positions by first row, and those rows
};

// Builds the plan from the full mesh's gather lists, the boundary nodes
// (0-based, any order) and the electrodes / sink.  Returns 0, or errnr 3
// when the split is unusable (no interior or no boundary node, or m above
// SCHUR_MMAX).
int schur_plan_host(const AssemblyLists& full, int n, const std::vector<int>& gamma_nodes,
                    const std::vector<int>& enr0, int lsink, int nsink0, SchurHost& out, int R = SCHUR_MS_R);

// Device arguments of the Schur kernels (one context's plan).
struct SchurArgs {
    int nI, m, L, K, ncol, mbI, WI, nblk, ncpl, ngg;
    int k0, nk;              // wavenumbers k0 .. k0 + nk - 1 of a launch (transpose .. back)
    int R;                   // columns per block of the forward sweep (16: two CTAs per SM, 32: one)
    const int *permI, *gam, *posI_src, *posG_src;
    int posI_sink, posG_sink, lsink;
    const int *gi_ptr, *gi_pos, *gi_ent, *gi_g;
    const int *gg_g, *gg_h, *gg_ent;
    const int *col_order, *blk_start;
    const int *bd_ptr, *bd_col, *bd_ent;
    int grp, ngrp;           // iterative Schur solve: electrodes per reference factor, groups
    int nbd;                 // entries of the boundary rows (bd_ptr[m])
    const int* first;        // [ncol] first non-zero interior row of column c
    const int* gsort;        // [m] boundary positions ordered by their column's first row
    const int* gfirst;       // [m] first row of gsort[q]'s column
    int* status;             // [K * L] errnr per (k, l); the interior factor uses [0, K)
    // forward sweep concurrent with the interior factor: progress[k] as
    // published by k_band_factor_blk (columns [0, progress[k]) final), or null
    const int* progress = nullptr;
};

// Right-hand sides of the interior solves, X[k][c][i] (zeroed by the
// caller), scaled by the interior factor's fak (so after the preparation
// pass): fak_i (+1 at the source's interior row, -1 at the sink's) in
// columns c < L, fak_i a(i, g) of A_IG in columns L + g; the unscaled
// coupling values a(g, i) also into cval[k][q].
template <typename T>
void launch_schur_rhs(const SchurArgs& s, const BandArgs<T>& full, const double* fakws, T* X, T* cval,
                      cudaStream_t st);
// Reversed row-packed copy of the interior factors for the back sweep:
// Lrev[k][c'][d] = L(n-1-c', n-1-c'-d), so that L^T in reversed numbering
// is lower-triangular banded with the forward sweep's layout.
template <typename T>
void launch_schur_transpose(const SchurArgs& s, const T* Lws, T* Lrev, cudaStream_t st);
// Forward sweep: X <- L^-1 X in place for every column (u^ = L^-1 F r_I,
// V^ = L^-1 F A_IG), each column block from its first non-zero row.
template <typename T>
void launch_schur_forward(const SchurArgs& s, const T* Lws, T* X, cudaStream_t st);
// waits (one thread, bounded) until `want` CTAs of a concurrent factor have begun
void launch_wait_started(const int* started, int want, int* status, cudaStream_t st);
// Gram products C[k][c][g] = sum_i V^[i][g] X[i][c] (c < L: A_GI w_l;
// c >= L: the lower triangle of A_GI Y = -S0), column-major with m rows.
template <typename T>
void launch_schur_gram(const SchurArgs& s, const T* X, T* C, cudaStream_t st);
// Systems sys0 .. sys0+nsys-1 (sys = k L + l): S_l = A_GG(l) - C_VV[k]
// into the workspace Sws[b] (m x m each), its Cholesky factor in place, and
// the boundary potentials xg[sys][g] = S_l^-1 (r_G - C[k][l]).
template <typename T>
void launch_schur_chol(const SchurArgs& s, const BandArgs<T>& full, const T* C, T* Sws, T* xg, int sys0, int nsys,
                       cudaStream_t st);
// Iterative form of the Schur solves (replaces launch_schur_chol).  Per
// wavenumber S_l = S0 + D_l, S0 = A_GG^area - V^T V^ (electrode independent),
// D_l the mixed-boundary part.  launch_schur_s0 forms S0 (full, column-major,
// [k][m][m]); launch_schur_ref factors one reference S0 + mean_{l in group}
// D_l per (k, group of s.grp electrodes) into Lref[(k ngrp + g)][m][m];
// launch_schur_iter solves every S_l p_G = r_G - C[k][l] by the preconditioned
// iteration x += S_ref^-1 (b - S_l x) until the correction is below tol
// |x|_inf, at most maxit steps; systems that do not get there are counted
// in nonconv[0] (device memory, two ints zeroed by the caller; nonconv[1]
// sums the iterations of the converged systems), and the caller then solves
// them all by the per-system Cholesky instead.
template <typename T>
void launch_schur_s0(const SchurArgs& s, const BandArgs<T>& full, const T* C, T* S0, cudaStream_t st);
template <typename T>
void launch_schur_ref(const SchurArgs& s, const BandArgs<T>& full, const T* S0, T* Lref, int* nonconv,
                      cudaStream_t st);
// Shared memory of the iteration's CTA (X and Z for SCHUR_IT_NS systems).
template <typename T> size_t schur_iter_smem(int m);
// Dv[(k L + l) nbd + q] = the mixed-boundary value of boundary-row entry q
// (bd_*) for electrode l at wavenumber k (nbd = bd_ptr[m]).
template <typename T>
void launch_schur_dvals(const SchurArgs& s, const BandArgs<T>& full, T* Dv, cudaStream_t st);
template <typename T>
void launch_schur_iter(const SchurArgs& s, const BandArgs<T>& full, const T* C, const T* S0, const T* Lref,
                       const T* Dv, T* xg, int maxit, double tol, int* nonconv, cudaStream_t st);

// z^_l = u^_l - V^ p_G (in place on the columns l < L of X).
template <typename T>
void launch_schur_zrebuild(const SchurArgs& s, T* X, const T* xg, cudaStream_t st);
// Back sweep L^T x^ = z^ of the columns l < L with the reversed factor,
// kpot(node, l, k) = fak x^ on the interior rows and p_G on the boundary
// rows (complex128 Fortran layout; real systems with zero imaginary parts).
template <typename T>
void launch_schur_back(const SchurArgs& s, const T* Lrev, const double* fakws, const T* X, const T* xg, int n,
                       cd* kpot, cudaStream_t st);
// Dynamic shared memory of a sweep for the interior band mbI with R columns.
template <typename T> size_t schur_sweep_smem(int mbI, int WI, int R);
