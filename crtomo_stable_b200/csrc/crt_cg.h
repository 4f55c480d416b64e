// crt_cg.h -- Gauss-Newton normal-equation CG (src/cg_mod.f90, src/update.f90).
#pragma once

#include "crt_common.cuh"

// Device-resident CG control block (cjgmod scalars).
struct CGState {
    double dr, dr0, dr1, alpha, beta;
    double gam;   // preconditioned form: Re(r^H z) of the last iteration head
    double num;   // numerator of alpha: dr (cjggra) or Re(r^H z) (preconditioned)
    double dr_chk; // |r|^2 at the last progress check of the learned correction
    int k;        // next iteration number (1-based)
    int done;     // 1 once the stop rule fired or ncgmax was reached
    int ncg;      // completed iterations
    int no_gnn;   // 1 once the learned correction has been switched off for this solve
    // the grid-wide form of the head and tail (one solve): arrivals at the
    // sums, the tail update being due, arrivals at the tail update, and the
    // head's choice of the base preconditioner's output
    int vcnt, pending, ucnt, use_base;
};

struct CGArgs {
    int M, N;             // manz, nanz
    int jmode;            // 0 complex J (cjggra), 1 real sensdc (ldc), 2 real part of complex J (lfpi)
    int jprec;            // storage of J: 0 FP64 (cd / double), 1 FP32 (cf / float); arithmetic is FP64
    int ltri, nx, nnb;    // regulariser: 0 five-point (smatm(M,3)), else neighbour list (smatm(M,nnb+1))
    int ncgmax;
    double lam, eps;
    const void* J;        // [M][N]: cd / cf (jmode 0/2) or double / float (jmode 1)
    const double* wd;     // [N] wmatd * wdfak
    const double* smatm;  // Fortran smatm(M, ncol)
    const int* nachbar;   // Fortran nachbar(M, nnb+1), 1-based, 0 = none
    double* cgfac;        // [M]
    cd* rhs;              // [M] scaled right-hand side (bvec on entry to cjg)
    cd *p, *r, *bvec, *dpar, *ap;   // [M],[M],[M],[M],[N]: ap holds w o (J p) after the reduction
    cd* part;             // [nsplit][N] partial J*p sums
    int nsplit;
    double* cgres;        // [ncgmax + 2]
    CGState* st;
    // preconditioned form (pc = 1): z = S^-1 r from the block preconditioner,
    // rold the residual of the previous head (flexible beta)
    int pc;
    cd *z, *rold;
    // learned correction on top of the base preconditioner (pc_gnn = 1):
    // zb holds the base's output (nullptr: the identity, i.e. r)
    int pc_gnn;
    const cd* zb;
    // fused matvec (fused = 1, launch_cg_iterations): J p and J^H (w o J p)
    // from one read of J, see k_cg_fused
    int fused;
    int fper;                     // columns per CTA
    cd* fpart;                    // [CGF_Q][grid][CGF_R] per-CTA partial sums of a row block
    cd* fv;                       // [CGF_Q][CGF_R] w o (J p) of a row block
    int* fcnt;                    // [CGF_Q] arrivals at a ring slot
    unsigned long long* fflag;    // [CGF_Q] ticket of the block whose w o (J p) a slot holds
    unsigned long long* fepoch;   // [1] advanced by every iteration tail (tickets stay unique)
    int* ferr;                    // [1] set when a wait gave up
    int flag_lag;                 // row blocks between a block's two uses (CGF_S .. CGF_Q - 1)
    double* vred;                 // [32][8] per-CTA partial sums of the grid-wide head and tail
};

// Fused matvec geometry: row blocks of CGF_R readings, a ring of CGF_Q
// reduction slots, CGF_S shared-memory stages of a CTA's J tile for each of
// the two uses of a block.
constexpr int CGF_R = 16, CGF_Q = 32, CGF_S = 2, CGF_NT = 512;
// dynamic shared memory of k_cg_fused for `per` columns per CTA
inline size_t cg_fused_smem(int per)
{
    return (size_t)2 * CGF_S * per * CGF_R * 8 + (size_t)per * 16 + (size_t)(CGF_NT / CGF_R) * CGF_R * 16 +
           CGF_R * 16;
}

// The learned correction is switched off for the rest of a solve when it
// yields a non-descent direction (Re r^H z <= 0) or when |r|^2 has not
// halved over GNN_GUARD_WINDOW iterations; the CG then restarts its
// direction from the base preconditioner.
constexpr int GNN_GUARD_WINDOW = 50;

struct SpcPlan;
struct Gnn;

// update.f90:63-231: cgfac and the scaled RHS from J, the data residual
// dat - sigmaa and the regularisation gradient lam * R * par.
void launch_cg_setup(const CGArgs& a, const cd* dat, const cd* sigmaa, const cd* par, cudaStream_t s);
// cjggra / cjggdc: resets the state, then runs up to `iters` iterations.
void launch_cg_init(const CGArgs& a, cudaStream_t s);
// pc = 1 applies the preconditioner before every head: the block factor
// `spc` (crt_spc.h), the learned correction `gnn` (crt_gnn.h) on top of it
// (zb holds the block result) or on top of the identity; either may be null.
void launch_cg_iterations(const CGArgs& a, int iters, const SpcPlan* spc, Gnn* gnn, cd* zb, cudaStream_t s);
// Whether the fused matvec can run for these arguments on `grid` CTAs of
// at most `smem_max` bytes of shared memory: complex64 J (jprec 1, jmode 0
// or 2) and the CTA's tile stages fitting.
bool cg_fused_fits(const CGArgs& a, int grid, size_t smem_max);
// update.f90:300-351: dpar *= cgfac (lfpi: (0, Re dpar) first), par += step
// dpar, bdpar = step * sum |dpar|^2.
void launch_cg_finish(const CGArgs& a, int lfpi, double step, cd* par, double* bdpar, cudaStream_t s);

// Several lambda candidates on one Jacobian.  Each lambda trial of the
// reference's inversion loop (src/inv.f90:769-912) runs update.f90 with
// cjggra / cjggdc on the same J; here up to CGL_MAX of them run side by side
// and the two matvecs of an iteration read every J entry once for all of
// them.  Candidate b keeps its vectors at offset b * M of the buffers in
// `a` (ap at b * N, the partial sums at b * nsplit * N, cgres at
// b * (ncgmax + 2), z and rold at b * M) and its control block at st + b;
// `a.lam` is unused.  `slot` maps the nl positions of a launch to
// candidates, so that the candidates still iterating can be compacted into
// fewer positions once others have stopped (set-up, init and finish take
// every candidate with the identity map).  Jacobi form (pc = 0, launch_cgl_iterations) or the
// block-preconditioned form (pc = 1, launch_cgl_iteration_pc after the
// caller has applied each candidate's preconditioner into its z; the
// learned correction is not batched).  Every candidate's arithmetic is the
// single solve's, in the same order.
constexpr int CGL_MAX = 8;
struct CGLArgs {
    CGArgs a;
    int nl;                 // candidates taking part in the launch
    int slot[CGL_MAX];      // position -> candidate (buffer slot); the identity unless compacted
    double lam[CGL_MAX];    // per candidate (by slot)
};

void launch_cgl_setup(const CGLArgs& L, const cd* dat, const cd* sigmaa, const cd* par, cudaStream_t s);
void launch_cgl_init(const CGLArgs& L, cudaStream_t s);
// returns the number of kernel launches enqueued
int launch_cgl_iterations(const CGLArgs& L, int iters, cudaStream_t s);
// one preconditioned iteration (head, matvecs, tail) of every candidate;
// returns the number of kernel launches
int launch_cgl_iteration_pc(const CGLArgs& L, cudaStream_t s);
// par_out[b * M ...] = par_in + step * cgfac_b o dpar_b; bdpar[b] as crt_update
void launch_cgl_finish(const CGLArgs& L, int lfpi, double step, const cd* par_in, cd* par_out, double* bdpar,
                       cudaStream_t s);
