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
