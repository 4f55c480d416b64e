// crt_spc.h -- block-tridiagonal preconditioner for the Gauss-Newton CG.
//
// After the Jacobi scaling of src/update.f90:200-231 (cgfac), the CG
// operator is  A = C J^H W J C + lam C R C  with C = diag(cgfac).  Its
// sparse part
//     S = diag(C_j^2 sum_i w_i |J_ij|^2) + lam C R C
// has a unit diagonal (that is what cgfac normalises) and the sparsity of
// the roughness operator R (bp / bptri, src/cg_mod.f90:547-613).  For the
// smoothness regularisers at the first Gauss-Newton steps lam R dominates
// the conditioning, so S^-1 is a strong preconditioner; the dense low-rank
// part J^H W J is left to the CG.
//
// S is ordered by reverse Cuthill-McKee on the element adjacency graph.
// With half-bandwidth b the permuted matrix is block tridiagonal in blocks
// of B = roundup(b, 32) rows:  diagonal blocks D_q and sub-diagonal blocks
// F_q (rows of block q, columns of block q-1).  The block LDL^T recurrence
//     T_0 = D_0,  T_q = D_q - F_q T_{q-1}^-1 F_q^T
// is run in FP32 with explicit inverses, which turns both triangular sweeps
// of an application into dense GEMVs:
//     u_q = T_q^-1 r_q                       (all blocks in parallel)
//     h_0 = u_0,  h_q = u_q - G_q h_{q-1},   G_q = T_q^-1 F_q
//     x_last = h_last,  x_q = h_q - H_q x_{q+1},  H_q = T_q^-1 F_{q+1}^T
// The preconditioner is FP32 and therefore not exactly linear; the CG that
// uses it takes the flexible (Polak-Ribiere) beta and keeps the reference's
// stop rule on the true residual |r|^2 <= eps |r0|^2.
//
// Segmented form (B <= 128, nb >= 32): the block chain is cut into nseg
// segments; the last block of each segment but the last is a separator.
// The segments' interiors I_p are factored side by side (one CTA each), the
// spikes V_p = A_Ip^-1 E_first F_{s_p} and W_p = A_Ip^-1 E_last F_{e_p}^T
// are formed by chains of block products, and the separators' Schur
// complement (block tridiagonal, nseg - 1 blocks)
//     Sd_p = D_{e_p} - F_{e_p} W_p[e_p - 1] - F_{e_p+1}^T V_{p+1}[e_p + 1]
//     So_p = - F_{e_p} V_p[e_p - 1]          (row c_p, column c_{p-1})
// is factored by the same recurrence.  An application solves the interiors
// side by side (y = A_I^-1 r_I), the separators from
// g_p = r_{c_p} - F_{e_p} y[e_p - 1] - F_{e_p+1}^T y[e_p + 1], and corrects
// the interiors, x_q = y_q - V_p[q] x_{c_{p-1}} - W_p[q] x_{c_p}, all blocks
// in parallel.  The result is S^-1 r as for the single chain (another
// elimination order, the same FP32 arithmetic per block); the sequential
// chains shrink from nb block steps to about nb / nseg + nseg.
#pragma once

#include <string>

#include "crt_common.cuh"

struct CGState;

struct SpcPlan {
    int ok = 0;            // plan built and usable
    int M = 0, B = 0, nb = 0, Mp = 0, bw = 0;
    int nent = 0;
    int* d_perm = nullptr;     // [Mp] permuted position -> element (-1: padding)
    int4* d_ent = nullptr;     // [nent] {dst in DF, i, j, smatm index}
    float* d_DF = nullptr;     // [2][nb][B][B]: D_q (T_q^-1 after the factor), F_q^T
    float* d_G = nullptr;      // [nb][B][B]  T_q^-1 F_q       (q >= 1)
    float* d_H = nullptr;      // [nb][B][B]  T_q^-1 F_{q+1}^T (q < nb-1)
    cf* d_h = nullptr;         // [Mp] sweep vector
    int* d_flag = nullptr;     // [1] 0 ok, else 1 + block of the first non-positive pivot
    // segmented form (nseg = 0: the single chain)
    int nseg = 0, nc = 0;
    int2* d_seg = nullptr;     // [nseg] first and last interior block of each segment (shared by clones)
    int* d_bseg = nullptr;     // [nb] segment of an interior block, -(1 + p) for separator p (shared)
    int* d_sep = nullptr;      // [nc] block of separator p (shared)
    float* d_V = nullptr;      // [nb][B][B] row-major, left spikes (interior blocks of segments p >= 1)
    float* d_W = nullptr;      // [nb][B][B] row-major, right spikes (segments p < nseg - 1)
    float* d_DFc = nullptr;    // [2][nc][B][B] separators' Schur complement: Sd_p, So_p^T
    float* d_Gc = nullptr;     // [nc][B][B] its G (column-major)
    float* d_Hc = nullptr;     // [nc][B][B] its H (column-major)
    cf* d_hc = nullptr;        // [nc B] separators' sweep vector
};

constexpr int SPC_MAX_B = 192;

// Host: reverse Cuthill-McKee ordering of the regulariser's graph, the block
// size and the assembly entry lists; allocates the device buffers.  Returns
// 0 on success; on a bandwidth above SPC_MAX_B the plan is left unusable
// (ok = 0) with the reason in `why`, which is not an error.
int spc_plan_build(SpcPlan& P, int M, int ltri, int nx, int nnb, const double* smatm, const int* nachbar,
                   std::string& why);
void spc_plan_free(SpcPlan& P);
// A plan with its own factor buffers (D/F, G, H, sweep vector, flag) that
// shares `src`'s ordering and entry list (device pointers included), for a
// second factor of the same S pattern (another lambda).  Freed with
// spc_plan_free_clone, before `src` is freed.
int spc_plan_clone(const SpcPlan& src, SpcPlan& dst);
void spc_plan_free_clone(SpcPlan& P);

// Assembles S from cgfac, lam and the device copy of smatm, and factors it.
void launch_spc_factor(const SpcPlan& P, const double* cgfac, const double* smatm, double lam, cudaStream_t s);
// z = S^-1 r (skipped once the CG state reports done).
void launch_spc_apply(const SpcPlan& P, const cd* r, cd* z, const CGState* st, cudaStream_t s);
