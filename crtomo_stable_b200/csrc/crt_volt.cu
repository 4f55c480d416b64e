// crt_volt.cu -- inverse Fourier transform over wavenumbers and voltages.
//
// k_hpot_electrodes : hpot(enr(p), c) for every pair of electrodes p, c --
//   the only potentials bvolti / bvolt read (src/rtrafo.f90:73-88 restricted
//   to electrode nodes): sum_k kwnwi(k) kpot(enr(p), c, k) / pi, FP64, in
//   the reference's k order.
// k_voltages : four-pole superposition of src/bvolti.f90:43-89 /
//   src/bvolt.f90:40-79 with the strnr/vnr decoding (C1 + 10000 C2).
// k_hpot_full : hpot for all nodes (CRMod potential output, bpot).
#include "crt_volt.h"

__global__ void k_hpot_electrodes(VoltArgs A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.L * A.L) return;
    const int p = t % A.L, c = t / A.L;     // potential electrode p, current electrode c
    const int node = A.enr0[p];
    cd s{0.0, 0.0};
    if (A.swrtr == 0) {
        s = A.kpot[(size_t)c * A.n + node];
    } else {
        for (int k = 0; k < A.K; ++k) s += A.kpot[((size_t)k * A.L + c) * A.n + node] * A.kwnwi[k];
        s = s / A.pi;
    }
    A.hel[(size_t)c * A.L + p] = s;
}

__device__ __forceinline__ cd hel_term(const VoltArgs& A, int ep, int ec)
{
    // min0(ep,1)*min0(ec,1) * hpot(enr(max0(ep,1)), max0(ec,1))
    double f = (double)(min(ep, 1) * min(ec, 1));
    const int p = max(ep, 1) - 1, c = max(ec, 1) - 1;
    return A.hel[(size_t)c * A.L + p] * f;
}

__global__ void k_voltages(VoltArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.N) return;
    const int s = A.strnr[i], v = A.vnr[i];
    const int e1 = s % 10000, e2 = (s - e1) / 10000, e3 = v % 10000, e4 = (v - e3) / 10000;
    cd d1 = hel_term(A, e4, e2), d2 = hel_term(A, e4, e1);
    cd d3 = hel_term(A, e3, e2), d4 = hel_term(A, e3, e1);
    cd volt = (d1 - d2) - (d3 - d4);
    if (A.ldc) volt = cd{volt.x, 0.0};
    A.volt[i] = volt;
    if (A.mode == 0) {
        // bvolti: sigmaa = -log(V), errnr 82 on a zero voltage
        double m = hypot(volt.x, volt.y);
        if (m == 0.0) {
            atomicMax(A.status, (int)CRT_ERR_ZERO_VOLT);
            A.sigmaa[i] = cd{0.0, 0.0};
        } else {
            A.sigmaa[i] = cd{-log(m), -atan2(volt.y, volt.x)};
        }
    } else {
        // bvolt: sigmaa = kfak * V
        double kf = A.kfak ? A.kfak[i] : 1.0;
        A.sigmaa[i] = volt * kf;
    }
}

__global__ void k_hpot_full(VoltArgs A, cd* hpot)
{
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)A.n * A.L) return;
    const int j = (int)(t % A.n), l = (int)(t / A.n);
    cd s{0.0, 0.0};
    if (A.swrtr == 0) {
        s = A.kpot[(size_t)l * A.n + j];
    } else {
        for (int k = 0; k < A.K; ++k) s += A.kpot[((size_t)k * A.L + l) * A.n + j] * A.kwnwi[k];
        s = s / A.pi;
    }
    hpot[(size_t)l * A.n + j] = s;
}

void launch_voltages(const VoltArgs& a, cudaStream_t st)
{
    int nel = a.L * a.L;
    k_hpot_electrodes<<<(nel + 255) / 256, 256, 0, st>>>(a);
    k_voltages<<<(a.N + 255) / 256, 256, 0, st>>>(a);
}

void launch_hpot_full(const VoltArgs& a, cd* hpot, cudaStream_t st)
{
    size_t tot = (size_t)a.n * a.L;
    k_hpot_full<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(a, hpot);
}
