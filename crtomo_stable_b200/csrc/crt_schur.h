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
//     [ A_GI   A_GG(l) ] [p_G] = [r_G]        r = e_src(l) - e_sink,
//
// gives p_I = w_l - Y p_G with w_l = A_II^-1 r_I, Y = A_II^-1 A_IG, and
// S_l p_G = r_G - A_GI w_l with the Schur complement S_l = A_GG(l) - A_GI Y.
// Per wavenumber: one band factorisation of A_II (the same prepared,
// scaled, unconjugated L L^T kernels as the direct path) and a multi-RHS
// band solve of the L + m columns [r_I | A_IG]; per (k, l): a dense m x m
// complex-symmetric Cholesky of S_l and the rebuild of p_I by a GEMM.  The
// arithmetic is FP64 (complex128 or real) throughout; the result equals the
// reference's per-system elimination up to rounding (same matrix, a
// different elimination order).
#pragma once

#include <vector>

#include "crt_band.h"
#include "crt_setup.h"

// Largest boundary set the dense Schur kernels take (panel in shared memory).
constexpr int SCHUR_MMAX = 768;
// Columns per CTA of the multi-RHS band solve and its column block.
constexpr int SCHUR_MS_R = 32;
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
    // multi-RHS solve: columns ordered by their first non-zero interior
    // row; blocks of SCHUR_MS_R columns and their first rows
    std::vector<int> col_order, blk_start;
};

// Builds the plan from the full mesh's gather lists, the boundary nodes
// (0-based, any order) and the electrodes / sink.  Returns 0, or errnr 3
// when the split is unusable (no interior or no boundary node, or m above
// SCHUR_MMAX).
int schur_plan_host(const AssemblyLists& full, int n, const std::vector<int>& gamma_nodes,
                    const std::vector<int>& enr0, int lsink, int nsink0, SchurHost& out);

// Device arguments of the Schur kernels (one context's plan).
struct SchurArgs {
    int nI, m, L, K, ncol, mbI, WI, nblk, ncpl, ngg;
    const int *permI, *gam, *posI_src, *posG_src;
    int posI_sink, posG_sink, lsink;
    const int *gi_ptr, *gi_pos, *gi_ent, *gi_g;
    const int *gg_g, *gg_h, *gg_ent;
    const int *col_order, *blk_start;
    int* status;             // [K * L] errnr per (k, l); the interior factor uses [0, K)
};

// Right-hand sides of the multi-RHS solve, X[k][c][i] (zeroed by the
// caller): +1 at the source's interior row and -1 at the sink's (columns
// c < L), the couplings a(i, g) of A_IG (columns L + g, also kept in
// cval[k][q] for the later steps).
template <typename T>
void launch_schur_rhs(const SchurArgs& s, const BandArgs<T>& full, T* X, T* cval, cudaStream_t st);
// Forward and back substitution with the interior factors (Lws, fakws as
// the band kernels leave them, column stride WI) of every column: X is
// overwritten by A_II^-1 X.  Uses the plan's column order and block starts.
template <typename T>
void launch_schur_msolve(const SchurArgs& s, const T* Lws, size_t lstride, const double* fakws, T* X,
                         cudaStream_t st);
// S0[k] = -A_GI Y (lower triangle, column-major m x m) for every k.
template <typename T>
void launch_schur_s0(const SchurArgs& s, const T* X, const T* cval, T* S0, cudaStream_t st);
// Systems sys0 .. sys0+nsys-1 (sys = k L + l): S_l = S0[k] + A_GG(l) into
// the workspace Sws[b] (m x m each), its Cholesky factor in place, and the
// boundary potentials xg[sys][g] = S_l^-1 (r_G - A_GI w_l).
template <typename T>
void launch_schur_chol(const SchurArgs& s, const BandArgs<T>& full, const T* S0, const T* X, const T* cval,
                       T* Sws, T* xg, int sys0, int nsys, cudaStream_t st);
// kpot(node, l, k) for every node: p_I = w_l - Y p_G on the interior rows,
// p_G on the boundary rows (complex128 Fortran layout; real systems with
// zero imaginary parts).
template <typename T>
void launch_schur_out(const SchurArgs& s, const T* X, const T* xg, int n, cd* kpot, cudaStream_t st);
// Dynamic shared memory of the multi-RHS solve for the interior band mbI.
template <typename T> size_t schur_msolve_smem(int mbI, int WI);
