// crt_sens.h -- reciprocity Jacobian (bsensi / bsendc / bsens).
#pragma once

#include "crt_common.cuh"

struct SensArgs {
    int n, E, L, K, N, nmn, maxnodes, swrtr;
    int mode;              // 0 bsensi (complex, sigma/V), 1 bsendc (real), 2 bsens (CRMod, -strom)
    int kchunk;            // wavenumbers staged per pass
    int out_prec;          // 0: store sens in FP64 (cd / double), 1: in FP32 (cf / float)
    double pi;
    const cd* kpt;         // [K][n][L]
    const double* elbg;    // [K][E][nmn]
    const double* kwnwi;   // [K]
    const int* nrel0;      // [ntot][maxnodes]
    const int* enk;        // [E]
    const int4* elec;      // [N] 0-based C1, C2, P1, P2 (-1 absent)
    const cd* sigma;       // [E]
    const cd* volt;        // [N]
    const double* strom;   // [N] or NULL
    void* sens;            // [E][N]: complex for modes 0/2, real for mode 1 (precision out_prec)
    cd* part;              // [E][N] partial sums when K is split (kchunk < K)
    cd* rfac;              // [N] scratch of the Gram form: each reading's factor, the divisions done once
};

void launch_transpose_kpot(const cd* kpot, cd* kpt, int n, int L, int K, cudaStream_t st);
size_t sens_smem(int L, int K, int nkmax, int nmn, int* kchunk, size_t limit, bool real);
void launch_sens(const SensArgs& a, size_t smem, bool real, cudaStream_t st);
// Gram form (crt_sens.cu): false when the electrodes or element nodes
// exceed its limits (L <= 168 for complex potentials, nk <= 4); then the
// per-reading kernel above is used.
bool sens_gram_plan(int L, int K, int nkmax, bool real, int* LP, int* kc, size_t* smem, int* nt);
void launch_sens_gram(const SensArgs& a, int LP, int kc, size_t smem, int nt, bool real, cudaStream_t st);
