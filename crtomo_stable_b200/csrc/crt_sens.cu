// crt_sens.cu -- reciprocity sensitivities (Jacobian).
//
// sens(i, e) = [sum_k w_k sum_{mi,mj} elbg(e,imn,k) dC(mj) dP(mi)] / pi * f
// with dC = kpot(., C2, k) - kpot(., C1, k) at the element nodes and
// dP = kpot(., P2, k) - kpot(., P1, k) (src/bsensi.f90:98-186), and
//   f = sigma_e / V_i            (bsensi, complex)
//   f = DBLE(sigma_e / V_i)      (bsendc, real potentials, src/bsendc.f90)
//   f = -strom_i                 (bsens, CRMod, src/bsens.f90:150-190)
//
// Layout: one CTA per area element.  The element's potentials for every
// wavenumber and electrode are staged in shared memory from the
// node-major transpose kpt[k][node][l] (coalesced 16-byte rows); each
// thread then owns one reading at a time and writes sens(i, e), which is
// contiguous in i (the Fortran sens(nanz, manz) layout).
#include "crt_sens.h"

__global__ void k_transpose_kpot(const cd* __restrict__ kpot, cd* __restrict__ kpt, int n, int L, int K)
{
    // kpot[(k*L + l)*n + j] -> kpt[(k*n + j)*L + l], 32x32 tiles per k.
    __shared__ cd tile[32][33];
    const int k = blockIdx.z;
    const int j0 = blockIdx.x * 32, l0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        int l = l0 + r, j = j0 + tx;
        if (l < L && j < n) tile[r][tx] = kpot[((size_t)k * L + l) * n + j];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int j = j0 + r, l = l0 + tx;
        if (l < L && j < n) kpt[((size_t)k * n + j) * L + l] = tile[tx][r];
    }
}

template <typename T>
__device__ __forceinline__ T ld_phi(const cd& v);
template <>
__device__ __forceinline__ double ld_phi<double>(const cd& v) { return v.x; }
template <>
__device__ __forceinline__ cd ld_phi<cd>(const cd& v) { return v; }

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_sens(SensArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int e = blockIdx.x;
    const int nk = A.enk[e];
    const int L = A.L, K = A.K, kc = A.kchunk;
    T* phi = reinterpret_cast<T*>(smem_raw);                // [kc][nk][L]
    double* ek = reinterpret_cast<double*>(phi + (size_t)kc * nk * L);   // [kc][nmn]
    const int tid = threadIdx.x;
    const cd sig = A.sigma[e];

    for (int k0 = 0; k0 < K; k0 += kc) {
        const int kn = min(kc, K - k0);
        __syncthreads();
        for (int t = tid; t < kn * nk * L; t += NT) {
            int l = t % L, m = (t / L) % nk, kk = t / (L * nk);
            int node = A.nrel0[e * A.maxnodes + m];
            phi[t] = ld_phi<T>(A.kpt[((size_t)(k0 + kk) * A.n + node) * L + l]);
        }
        for (int t = tid; t < kn * A.nmn; t += NT) {
            int kk = t / A.nmn, q = t % A.nmn;
            ek[t] = A.elbg[((size_t)(k0 + kk) * A.E + e) * A.nmn + q];
        }
        __syncthreads();
        for (int i = tid; i < A.N; i += NT) {
            const int4 el = A.elec[i];    // 0-based C1, C2, P1, P2; -1 when absent
            T acc = Sc<T>::zero();
            for (int kk = 0; kk < kn; ++kk) {
                const T* ph = phi + (size_t)kk * nk * L;
                const double* km = ek + kk * A.nmn;
                T h = Sc<T>::zero();
                for (int mi = 0; mi < nk; ++mi) {
                    const T* pm = ph + mi * L;
                    T s3 = el.z >= 0 ? pm[el.z] : Sc<T>::zero();
                    T s4 = el.w >= 0 ? pm[el.w] : Sc<T>::zero();
                    T dP = s4 - s3;
                    for (int mj = 0; mj < nk; ++mj) {
                        const T* pn = ph + mj * L;
                        T s1 = el.x >= 0 ? pn[el.x] : Sc<T>::zero();
                        T s2 = el.y >= 0 ? pn[el.y] : Sc<T>::zero();
                        const int imx = max(mi, mj), imn_ = min(mi, mj);
                        h += scale(Sc<T>::mul(s2 - s1, dP), km[imx * (imx + 1) / 2 + imn_]);
                    }
                }
                if (A.swrtr == 0) acc = h;
                else acc += scale(h, A.kwnwi[k0 + kk]);
            }
            const size_t o = (size_t)e * A.N + i;
            if (k0 > 0) acc += Sc<T>::from(*reinterpret_cast<const cd*>(&A.part[o]));
            if (k0 + kn < K) {
                A.part[o] = Sc<T>::to_cd(acc);
                continue;
            }
            // final scaling (FP64), stored in the requested precision
            cd res;
            if (A.mode == 0) {
                cd d = Sc<T>::to_cd(acc);
                if (A.swrtr != 0) d = d / A.pi;
                res = (d * sig) / A.volt[i];
            } else if (A.mode == 1) {
                double d = Sc<T>::to_cd(acc).x;
                if (A.swrtr != 0) d = d / A.pi;
                cd q = sig / A.volt[i];
                res = cd{d * q.x, 0.0};
            } else {
                cd d = Sc<T>::to_cd(acc);
                const double st = A.strom ? A.strom[i] : 1.0;
                if (A.swrtr == 0) d = d * st;
                else d = d * (st / A.pi);
                res = -d;
            }
            if (A.mode == 1) {
                if (A.out_prec) reinterpret_cast<float*>(A.sens)[o] = (float)res.x;
                else reinterpret_cast<double*>(A.sens)[o] = res.x;
            } else {
                if (A.out_prec) reinterpret_cast<cf*>(A.sens)[o] = cf{(float)res.x, (float)res.y};
                else reinterpret_cast<cd*>(A.sens)[o] = res;
            }
        }
    }
}

size_t sens_smem(int L, int K, int nkmax, int nmn, int* kchunk, size_t limit, bool real)
{
    const size_t tsz = real ? sizeof(double) : sizeof(cd);
    int kc = K;
    while (kc > 1 && (size_t)kc * nkmax * L * tsz + (size_t)kc * nmn * 8 > limit) --kc;
    *kchunk = kc;
    return (size_t)kc * nkmax * L * tsz + (size_t)kc * nmn * 8 + 32;
}

void launch_transpose_kpot(const cd* kpot, cd* kpt, int n, int L, int K, cudaStream_t st)
{
    dim3 grid((n + 31) / 32, (L + 31) / 32, K), block(32, 8);
    k_transpose_kpot<<<grid, block, 0, st>>>(kpot, kpt, n, L, K);
}

void launch_sens(const SensArgs& a, size_t smem, bool real, cudaStream_t st)
{
    constexpr int NT = 256;
    if (real) {
        cudaFuncSetAttribute(k_sens<double, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_sens<double, NT><<<a.E, NT, smem, st>>>(a);
    } else {
        cudaFuncSetAttribute(k_sens<cd, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_sens<cd, NT><<<a.E, NT, smem, st>>>(a);
    }
}
