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

#include <algorithm>

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

// ld_phi as an asynchronous copy into shared memory (cp.async): the whole
// complex value, or its real part (the first 8 bytes)
template <typename T>
__device__ __forceinline__ void phi_async(T* dst, const cd* src);
template <>
__device__ __forceinline__ void phi_async<cd>(cd* dst, const cd* src) { cp_async16(dst, src); }
template <>
__device__ __forceinline__ void phi_async<double>(double* dst, const cd* src)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(&src->x) : "memory");
}

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

// Gram form of the same sum.  With Phi_k the nk x L potentials of the
// element's nodes and E_k its element matrix,
//   G = sum_k w_k Phi_k^T E_k Phi_k      (L x L, symmetric: E_k is)
// holds G(a, b) = sum_{mi,mj} E_k(mi, mj) phi_a(mi) phi_b(mj) summed over the
// wavenumbers, and every reading is the four-term combination
//   G(P2,C2) - G(P2,C1) - G(P1,C2) + G(P1,C1)
// of the reciprocity sum of src/bsensi.f90:98-186 (the reference forms the
// potential differences first; the two orders agree to FP64 rounding of
// the products).  G is accumulated as a rank-(K nk) product: one thread per
// 4 x 4 tile of its lower triangle (small tiles: many warps per element),
// operands staged per chunk of
// wavenumbers (Phi_k and w_k E_k Phi_k), then written to shared memory for
// the readings' gathers.
constexpr int GR_TA = 4, GR_TB = 4;

__device__ __forceinline__ int gram_idx(int a, int b)
{
    if (a < b) {
        const int t = a;
        a = b;
        b = t;
    }
    return a * (a + 1) / 2 + b;
}

template <typename T, int MAXT>
__global__ void __launch_bounds__(MAXT) k_sens_gram(SensArgs A, int LP, int kc)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sbuf = reinterpret_cast<T*>(smem_raw);
    const int e = blockIdx.x;
    const int nk = A.enk[e];
    const int L = A.L, K = A.K;
    const int RB = LP / GR_TA, ntile = RB * (RB + 1) / 2;
    const int tid = threadIdx.x;
    // tile of this thread: row block R, column block Cb <= R
    int R = 0;
    while ((R + 1) * (R + 2) / 2 <= tid) ++R;
    const int Cb = tid - R * (R + 1) / 2;
    const bool has_tile = tid < ntile;
    T acc[GR_TA][GR_TB];
#pragma unroll
    for (int i = 0; i < GR_TA; ++i)
#pragma unroll
        for (int j = 0; j < GR_TB; ++j) acc[i][j] = Sc<T>::zero();
    T* phi = sbuf;                                   // [kc][nk][LP]
    // [kc][nk][GR_TB][LP / GR_TB]: column b at (b % GR_TB) LP/GR_TB + b / GR_TB,
    // so the tile loads of consecutive column blocks are consecutive words
    T* wu = sbuf + (size_t)kc * nk * LP;
    const int LQ = LP / GR_TB;
    // the element's nodes once, so the potential gathers below do not wait
    // on an index load each
    __shared__ int s_node[4];
    if (tid < nk) s_node[tid] = A.nrel0[e * A.maxnodes + tid];
    // flat index t = (kk nk + m) LP + a of the staging loops, stepped by the
    // block size without divisions: a += da, q = kk nk + m += dq (+ carry)
    const int da = blockDim.x % LP, dq = blockDim.x / LP;
    const int a_0 = tid % LP, q_0 = tid / LP;
    for (int k0 = 0; k0 < K; k0 += kc) {
        const int kn = min(kc, K - k0);
        const int tot = kn * nk * LP;
        __syncthreads();
        {
            // the potentials by cp.async (every copy of the thread in flight
            // at once; the real form takes the real parts, 8 bytes each)
            int a = a_0, m = q_0 % nk, kk = q_0 / nk;
            for (int t = tid; t < tot; t += blockDim.x) {
                if (a < L) phi_async<T>(phi + t, A.kpt + ((size_t)(k0 + kk) * A.n + s_node[m]) * L + a);
                else phi[t] = Sc<T>::zero();
                a += da;
                m += dq;
                if (a >= LP) {
                    a -= LP;
                    ++m;
                }
                while (m >= nk) {
                    m -= nk;
                    ++kk;
                }
            }
            cp_async_commit();
            cp_async_wait_all();
        }
        __syncthreads();
        {
            int b = a_0, m = q_0 % nk, kk = q_0 / nk;
            for (int t = tid; t < tot; t += blockDim.x) {
                const double* km = A.elbg + ((size_t)(k0 + kk) * A.E + e) * A.nmn;
                const double w = A.swrtr ? A.kwnwi[k0 + kk] : 1.0;
                T v = Sc<T>::zero();
                for (int m2 = 0; m2 < nk; ++m2) {
                    const int ix = max(m, m2), in = min(m, m2);
                    v += scale(phi[((size_t)kk * nk + m2) * LP + b], km[ix * (ix + 1) / 2 + in]);
                }
                wu[t - b + (b % GR_TB) * LQ + b / GR_TB] = scale(v, w);
                b += da;
                m += dq;
                if (b >= LP) {
                    b -= LP;
                    ++m;
                }
                while (m >= nk) {
                    m -= nk;
                    ++kk;
                }
            }
        }
        __syncthreads();
        if (has_tile) {
            for (int q = 0; q < kn * nk; ++q) {
                const T* pa = phi + (size_t)q * LP + R * GR_TA;
                const T* pb = wu + (size_t)q * LP + Cb;
                T av[GR_TA], bv[GR_TB];
#pragma unroll
                for (int i = 0; i < GR_TA; ++i) av[i] = pa[i];
#pragma unroll
                for (int j = 0; j < GR_TB; ++j) bv[j] = pb[j * LQ];
#pragma unroll
                for (int i = 0; i < GR_TA; ++i)
#pragma unroll
                    for (int j = 0; j < GR_TB; ++j) fms_acc(acc[i][j], -av[i], bv[j]);
            }
        }
    }
    __syncthreads();
    T* G = sbuf;   // lower triangle, packed
    if (has_tile) {
#pragma unroll
        for (int i = 0; i < GR_TA; ++i)
#pragma unroll
            for (int j = 0; j < GR_TB; ++j) {
                const int a = R * GR_TA + i, b = Cb * GR_TB + j;
                if (a >= b && a < L) G[a * (a + 1) / 2 + b] = acc[i][j];
            }
    }
    __syncthreads();
    const cd sig = A.sigma[e];
    // reading i: its four Gram entries, the reference's scaling, the store
    auto value = [&](int4 el, int i) {
        auto g = [&](int a, int b) { return (a < 0 || b < 0) ? Sc<T>::zero() : G[gram_idx(a, b)]; };
        const T acc_i = ((g(el.w, el.y) - g(el.w, el.x)) - g(el.z, el.y)) + g(el.z, el.x);
        cd res;
        if (A.out_prec) {
            // stored in FP32: each reading's divisions are done once
            // (k_sens_factors), which changes the FP64 value only by
            // rounding far below the stored precision
            const cd f = A.rfac[i];
            if (A.mode == 0) res = (Sc<T>::to_cd(acc_i) * f) * sig;
            else if (A.mode == 1) res = cd{Sc<T>::to_cd(acc_i).x * (sig * f).x, 0.0};
            else res = Sc<T>::to_cd(acc_i) * f.x;
        } else if (A.mode == 0) {
            // stored in FP64: the reference's operations in its order
            cd d = Sc<T>::to_cd(acc_i);
            if (A.swrtr != 0) d = d / A.pi;
            res = (d * sig) / A.volt[i];
        } else if (A.mode == 1) {
            double d = Sc<T>::to_cd(acc_i).x;
            if (A.swrtr != 0) d = d / A.pi;
            const cd q = sig / A.volt[i];
            res = cd{d * q.x, 0.0};
        } else {
            cd d = Sc<T>::to_cd(acc_i);
            const double st = A.strom ? A.strom[i] : 1.0;
            if (A.swrtr == 0) d = d * st;
            else d = d * (st / A.pi);
            res = -d;
        }
        return res;
    };
    auto store = [&](cd res, int i) {
        const size_t o = (size_t)e * A.N + i;
        if (A.mode == 1) {
            if (A.out_prec) reinterpret_cast<float*>(A.sens)[o] = (float)res.x;
            else reinterpret_cast<double*>(A.sens)[o] = res.x;
        } else {
            if (A.out_prec) reinterpret_cast<cf*>(A.sens)[o] = cf{(float)res.x, (float)res.y};
            else reinterpret_cast<cd*>(A.sens)[o] = res;
        }
    };
    // four readings per thread at a time: their (dependent) chains overlap
    const int nt = blockDim.x;
    for (int i0 = tid; i0 < A.N; i0 += 4 * nt) {
        int4 el[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = i0 + q * nt;
            el[q] = i < A.N ? A.elec[i] : make_int4(-1, -1, -1, -1);
        }
        cd res[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = i0 + q * nt;
            res[q] = i < A.N ? value(el[q], i) : cd{0.0, 0.0};
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i0 + q * nt < A.N) store(res[q], i0 + q * nt);
    }
}

// Each reading's factor of the Gram form's output for FP32 storage, so that
// the per-element loop multiplies where the reference divides: 1 / (V_i pi) for bsensi and
// bsendc (sigma / V_i scales the Gram sum; pi only with swrtr), -I_i / pi
// (or -I_i without swrtr) for bsens.
__global__ void k_sens_factors(SensArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.N) return;
    const double sp = A.swrtr != 0 ? 1.0 / A.pi : 1.0;
    cd f;
    if (A.mode == 0 || A.mode == 1) {
        f = (cd{1.0, 0.0} / A.volt[i]) * sp;
    } else {
        const double st = A.strom ? A.strom[i] : 1.0;
        f = cd{-st * sp, 0.0};
    }
    A.rfac[i] = f;
}

bool sens_gram_plan(int L, int K, int nkmax, bool real, int* LP_out, int* kc_out, size_t* smem_out, int* nt_out)
{
    const size_t tsz = real ? sizeof(double) : sizeof(cd);
    const int LP = (L + GR_TA - 1) / GR_TA * GR_TA;
    const int RB = LP / GR_TA, ntile = RB * (RB + 1) / 2;
    if (nkmax > 4 || ntile > 1024) return false;
    const size_t gbytes = (size_t)LP * (LP + 1) / 2 * tsz;
    const size_t limit = 200 * 1024;
    if (gbytes > limit) return false;
    int kc = K;
    while (kc > 1 && 2 * (size_t)kc * nkmax * LP * tsz > std::max(gbytes, (size_t)64 * 1024)) --kc;
    *LP_out = LP;
    *kc_out = kc;
    *smem_out = std::max(gbytes, 2 * (size_t)kc * nkmax * LP * tsz);
    *nt_out = (ntile + 31) / 32 * 32;
    return true;
}

void launch_sens_gram(const SensArgs& a, int LP, int kc, size_t smem, int nt, bool real, cudaStream_t st)
{
    // one thread per tile: 320 threads up to 76 electrodes, 576 up to 132
    if (a.out_prec) k_sens_factors<<<(a.N + 255) / 256, 256, 0, st>>>(a);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<a.E, nt, smem, st>>>(a, LP, kc);
    };
    if (real) {
        if (nt <= 320) go(k_sens_gram<double, 320>);
        else if (nt <= 576) go(k_sens_gram<double, 576>);
        else go(k_sens_gram<double, 1024>);
    } else {
        if (nt <= 320) go(k_sens_gram<cd, 320>);
        else if (nt <= 576) go(k_sens_gram<cd, 576>);
        else go(k_sens_gram<cd, 1024>);
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
