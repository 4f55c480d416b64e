// crt_volt.h -- wavenumber quadrature and four-pole voltages.
#pragma once

#include "crt_common.cuh"

struct VoltArgs {
    int n, L, K, N, swrtr, ldc;
    int mode;                 // 0: bvolti (-log V), 1: bvolt (kfak * V)
    double pi;
    const cd* kpot;           // kpot(sanz, eanz, kwnanz)
    const double* kwnwi;      // [K]
    const int* enr0;          // [L]
    const int *strnr, *vnr;   // [N]
    const double* kfak;       // [N] or NULL
    cd* hel;                  // [L][L] hpot at electrode nodes: hel[c*L + p]
    cd* volt;                 // [N]
    cd* sigmaa;               // [N]
    int* status;
};

void launch_voltages(const VoltArgs& a, cudaStream_t st);
void launch_hpot_full(const VoltArgs& a, cd* hpot, cudaStream_t st);
