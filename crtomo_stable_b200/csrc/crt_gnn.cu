// crt_gnn.cu -- learned correction of the CG preconditioner: inference,
// training (forward with stored activations, backward, Adam) and the
// residual/error records of the plain CG.  The network is described in
// crt_gnn.h.  One warp per model cell: lane c holds channel c of the cell's
// 32-wide state, and the 32 x 32 products run as shuffle broadcasts against
// weights staged in shared memory (the products are too narrow for the
// tensor cores to pay).  Weight gradients are summed per warp in registers,
// per CTA in shared memory and over CTAs by a fixed-order reduction, so
// training is deterministic.
#include "crt_gnn.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "crt_cg.h"

namespace {

constexpr int GT = 256;              // threads per CTA
constexpr int GWARPS = GT / 32;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float bf2f(unsigned short b) { return __uint_as_float((unsigned)b << 16); }

__device__ __forceinline__ float warp_sum_f(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Stage n bf16 weights from global into shared memory as FP32.
__device__ __forceinline__ void stage_w(float* dst, const unsigned short* src, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = bf2f(src[i]);
}

// Transposed copy of a 32 x 32 block: dst[c][k] = src[k][c].
__device__ __forceinline__ void stage_wt(float* dst, const unsigned short* src)
{
    for (int i = threadIdx.x; i < GNN_W * GNN_W; i += blockDim.x) {
        const int k = i / GNN_W, c = i % GNN_W;
        dst[c * (GNN_W + 1) + k] = bf2f(src[i]);
    }
}

__global__ void k_gnn_edges(const int* __restrict__ nbr, const int* __restrict__ nsm, const double* __restrict__ cgfac,
                            const double* __restrict__ smatm, double lam, float* a, int M)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= M * GNN_D) return;
    const int i = idx / GNN_D, j = nbr[idx];
    a[idx] = j >= 0 ? (float)(lam * cgfac[i] * smatm[nsm[idx]] * cgfac[j]) : 0.0f;
}

// s = 1 / rms(r) (0 for a zero residual), one CTA.
__global__ void k_gnn_norm(const cd* __restrict__ r, int M, double* scal, const CGState* st)
{
    __shared__ double red[32];
    if (st && (st->done || st->no_gnn)) return;
    double v = 0.0;
    for (int i = threadIdx.x; i < M; i += blockDim.x) v += cabs2(r[i]);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        scal[0] = t > 0.0 ? sqrt((double)M / t) : 0.0;
    }
}

// Features of an application: [r, base] * s.
__global__ void k_gnn_feat(const cd* __restrict__ r, const cd* __restrict__ zb, const double* __restrict__ scal,
                           float* x, int M, const CGState* st)
{
    if (st && (st->done || st->no_gnn)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const double s = scal[0];
    const cd ri = r[i], bi = zb ? zb[i] : ri;
    reinterpret_cast<float4*>(x)[i] = make_float4((float)(ri.x * s), (float)(ri.y * s), (float)(bi.x * s), (float)(bi.y * s));
}

// Features of a training record.
__global__ void k_gnn_feat_rec(const cf* __restrict__ xr, float* x, int M)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const cf a = xr[2 * i], b = xr[2 * i + 1];
    reinterpret_cast<float4*>(x)[i] = make_float4(a.x, a.y, b.x, b.y);
}

// h0 = tanh(Win^T x)
__global__ void __launch_bounds__(GT) k_gnn_in(const unsigned short* __restrict__ wb, const float* __restrict__ x,
                                               float* h0, int M, const CGState* st)
{
    __shared__ float w[GNN_F * GNN_W];
    if (st && (st->done || st->no_gnn)) return;
    stage_w(w, wb + GNN_OFF_IN, GNN_F * GNN_W);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float4 xi = reinterpret_cast<const float4*>(x)[i];
        float acc = w[0 * GNN_W + lane] * xi.x;
        acc = fmaf(w[1 * GNN_W + lane], xi.y, acc);
        acc = fmaf(w[2 * GNN_W + lane], xi.z, acc);
        acc = fmaf(w[3 * GNN_W + lane], xi.w, acc);
        h0[(size_t)i * GNN_W + lane] = tanhf(acc);
    }
}

// h_l = tanh(Ws^T h_{l-1} + Wn^T sum_j a_ij h_{l-1,j}); the aggregate is kept
// for the backward pass when agg != nullptr.
__global__ void __launch_bounds__(GT) k_gnn_layer(const unsigned short* __restrict__ wb, int l,
                                                  const float* __restrict__ hp, float* hn, float* agg,
                                                  const int* __restrict__ nbr, const float* __restrict__ a, int M,
                                                  const CGState* st)
{
    __shared__ float ws[GNN_W * GNN_W], wn[GNN_W * GNN_W];
    if (st && (st->done || st->no_gnn)) return;
    const unsigned short* base = wb + GNN_OFF_L + l * GNN_LSTRIDE;
    stage_w(ws, base, GNN_W * GNN_W);
    stage_w(wn, base + GNN_W * GNN_W, GNN_W * GNN_W);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float hv = hp[(size_t)i * GNN_W + lane];
        float m = 0.0f;
#pragma unroll
        for (int d = 0; d < GNN_D; ++d) {
            const int j = nbr[i * GNN_D + d];
            if (j >= 0) m = fmaf(a[i * GNN_D + d], hp[(size_t)j * GNN_W + lane], m);
        }
        if (agg) agg[(size_t)i * GNN_W + lane] = m;
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < GNN_W; ++k) {
            acc = fmaf(ws[k * GNN_W + lane], __shfl_sync(FULL, hv, k), acc);
            acc = fmaf(wn[k * GNN_W + lane], __shfl_sync(FULL, m, k), acc);
        }
        hn[(size_t)i * GNN_W + lane] = tanhf(acc);
    }
}

// z = base + (Wout^T h3) / s
__global__ void __launch_bounds__(GT) k_gnn_out_apply(const unsigned short* __restrict__ wb, const float* __restrict__ h3,
                                                      const cd* __restrict__ r, const cd* __restrict__ zb,
                                                      const double* __restrict__ scal, cd* z, int M, const CGState* st)
{
    if (st && (st->done || st->no_gnn)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float w0 = bf2f(wb[GNN_OFF_OUT + lane * GNN_O]), w1 = bf2f(wb[GNN_OFF_OUT + lane * GNN_O + 1]);
    const double s = scal[0], inv = s > 0.0 ? 1.0 / s : 0.0;
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float hv = h3[(size_t)i * GNN_W + lane];
        const float o0 = warp_sum_f(w0 * hv), o1 = warp_sum_f(w1 * hv);
        if (lane == 0) {
            const cd b = zb ? zb[i] : r[i];
            z[i] = cd{b.x + (double)o0 * inv, b.y + (double)o1 * inv};
        }
    }
}

// Block reduction of per-warp partials red[warp][n] into part[blk][off + idx].
__device__ void block_partials(float* red, int n, float* part, int off)
{
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        float v = 0.0f;
        for (int w = 0; w < GWARPS; ++w) v += red[w * n + q];
        part[(size_t)blockIdx.x * GNN_NPARAM + off + q] = v;
    }
}

// Output layer of a record: loss, dL/dout = 2 (out - t) / |t|^2, gradient of
// Wout and du3 = (Wout dout) o (1 - h3^2).
__global__ void __launch_bounds__(GT) k_gnn_out_loss(const unsigned short* __restrict__ wb, const float* __restrict__ h3,
                                                     const cf* __restrict__ t, float tinv, float* du, float* part,
                                                     double* loss, int M)
{
    extern __shared__ float red[];   // [GWARPS][W * O]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float w0 = bf2f(wb[GNN_OFF_OUT + lane * GNN_O]), w1 = bf2f(wb[GNN_OFF_OUT + lane * GNN_O + 1]);
    float g0 = 0.0f, g1 = 0.0f, lsum = 0.0f;
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float hv = h3[(size_t)i * GNN_W + lane];
        const float o0 = warp_sum_f(w0 * hv), o1 = warp_sum_f(w1 * hv);
        const cf ti = t[i];
        const float e0 = o0 - ti.x, e1 = o1 - ti.y;
        lsum += e0 * e0 + e1 * e1;
        const float d0 = 2.0f * e0 * tinv, d1 = 2.0f * e1 * tinv;
        g0 = fmaf(hv, d0, g0);
        g1 = fmaf(hv, d1, g1);
        const float dh = w0 * d0 + w1 * d1;
        du[(size_t)i * GNN_W + lane] = dh * (1.0f - hv * hv);
    }
    red[warp * GNN_W * GNN_O + lane * GNN_O] = g0;
    red[warp * GNN_W * GNN_O + lane * GNN_O + 1] = g1;
    block_partials(red, GNN_W * GNN_O, part, GNN_OFF_OUT);
    if (lane == 0) atomicAdd(loss, (double)(lsum * tinv));   // every lane holds the warp's full sum
}

// Backward of layer l, part A (per cell i): gradients of Ws and Wn from du_i,
// the self term Ws du_i into dhp and dm_i = Wn du_i in place of the
// aggregate.
__global__ void __launch_bounds__(GT) k_gnn_bwd_a(const unsigned short* __restrict__ wb, int l,
                                                  const float* __restrict__ hp, float* agg, const float* __restrict__ du,
                                                  float* dhp, float* part, int M)
{
    extern __shared__ float sm[];
    float* wst = sm;                               // [W][W+1] Ws transposed
    float* wnt = wst + GNN_W * (GNN_W + 1);        // [W][W+1] Wn transposed
    float* red = wnt + GNN_W * (GNN_W + 1);        // [GWARPS][2 W W]
    const unsigned short* base = wb + GNN_OFF_L + l * GNN_LSTRIDE;
    stage_wt(wst, base);
    stage_wt(wnt, base + GNN_W * GNN_W);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float as[GNN_W], an[GNN_W];
#pragma unroll
    for (int k = 0; k < GNN_W; ++k) {
        as[k] = 0.0f;
        an[k] = 0.0f;
    }
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float u = du[(size_t)i * GNN_W + lane];        // lane = output channel c
        const float hv = hp[(size_t)i * GNN_W + lane];
        const float mv = agg[(size_t)i * GNN_W + lane];
        float ds = 0.0f, dm = 0.0f;
#pragma unroll
        for (int k = 0; k < GNN_W; ++k) {
            as[k] = fmaf(__shfl_sync(FULL, hv, k), u, as[k]);   // dWs[k][c]
            an[k] = fmaf(__shfl_sync(FULL, mv, k), u, an[k]);   // dWn[k][c]
            const float uk = __shfl_sync(FULL, u, k);           // du[c = k]
            ds = fmaf(wst[k * (GNN_W + 1) + lane], uk, ds);      // lane = input k': sum_c Ws[k'][c] du[c]
            dm = fmaf(wnt[k * (GNN_W + 1) + lane], uk, dm);
        }
        dhp[(size_t)i * GNN_W + lane] = ds;
        agg[(size_t)i * GNN_W + lane] = dm;
    }
#pragma unroll
    for (int k = 0; k < GNN_W; ++k) {
        red[warp * 2 * GNN_W * GNN_W + k * GNN_W + lane] = as[k];
        red[warp * 2 * GNN_W * GNN_W + GNN_W * GNN_W + k * GNN_W + lane] = an[k];
    }
    block_partials(red, 2 * GNN_W * GNN_W, part, GNN_OFF_L + l * GNN_LSTRIDE);
}

// Backward of layer l, part B (per cell j): dh_{l-1,j} = self term +
// sum_i a_ij dm_i over the cells i that list j, then du_{l-1} = dh o (1 - h^2).
__global__ void __launch_bounds__(GT) k_gnn_bwd_b(const float* __restrict__ hp, const float* __restrict__ dm,
                                                  float* dhp, const int* __restrict__ nbr, const int* __restrict__ rev,
                                                  const float* __restrict__ a, int M)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = blockIdx.x * GWARPS + warp; j < M; j += gridDim.x * GWARPS) {
        float d = dhp[(size_t)j * GNN_W + lane];
#pragma unroll
        for (int q = 0; q < GNN_D; ++q) {
            const int i = nbr[j * GNN_D + q];
            if (i >= 0) d = fmaf(a[i * GNN_D + rev[j * GNN_D + q]], dm[(size_t)i * GNN_W + lane], d);
        }
        const float hv = hp[(size_t)j * GNN_W + lane];
        dhp[(size_t)j * GNN_W + lane] = d * (1.0f - hv * hv);
    }
}

// Gradient of Win from du0 and the features.
__global__ void __launch_bounds__(GT) k_gnn_bwd_in(const float* __restrict__ x, const float* __restrict__ du, float* part,
                                                   int M)
{
    __shared__ float red[GWARPS * GNN_F * GNN_W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float g[GNN_F] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int i = blockIdx.x * GWARPS + warp; i < M; i += gridDim.x * GWARPS) {
        const float u = du[(size_t)i * GNN_W + lane];
        const float4 xi = reinterpret_cast<const float4*>(x)[i];
        g[0] = fmaf(xi.x, u, g[0]);
        g[1] = fmaf(xi.y, u, g[1]);
        g[2] = fmaf(xi.z, u, g[2]);
        g[3] = fmaf(xi.w, u, g[3]);
    }
#pragma unroll
    for (int f = 0; f < GNN_F; ++f) red[warp * GNN_F * GNN_W + f * GNN_W + lane] = g[f];
    block_partials(red, GNN_F * GNN_W, part, GNN_OFF_IN);
}

// g[p] += scale * sum over CTAs of part[b][p] (fixed order).
__global__ void k_gnn_reduce(const float* __restrict__ part, int nblk, float scale, float* g)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= GNN_NPARAM) return;
    float v = 0.0f;
    for (int b = 0; b < nblk; ++b) v += part[(size_t)b * GNN_NPARAM + p];
    g[p] += scale * v;
}

__global__ void k_gnn_round(const float* __restrict__ w, unsigned short* wb)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < GNN_NPARAM) wb[p] = __bfloat16_as_ushort(__float2bfloat16_rn(w[p]));
}

__global__ void k_gnn_adam(float* w, float* m, float* v, float* g, unsigned short* wb, float lr, float b1c, float b2c)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= GNN_NPARAM) return;
    const float gp = g[p];
    const float mp = 0.9f * m[p] + 0.1f * gp;
    const float vp = 0.999f * v[p] + 0.001f * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float wp = w[p] - lr * (mp / b1c) / (sqrtf(vp / b2c) + 1e-8f);
    w[p] = wp;
    g[p] = 0.0f;
    wb[p] = __bfloat16_as_ushort(__float2bfloat16_rn(wp));
}

// Record of one iterate: x = [r s, b s], t = (xs - xk - b) s, |t|^2 into scal[2].
__global__ void k_gnn_make_rec(const cd* __restrict__ rk, const cd* __restrict__ bk, const cd* __restrict__ xk,
                               const cd* __restrict__ xs, double* scal, cf* x, cf* t, int M)
{
    __shared__ double red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < M) {
        const double s = scal[0];
        const cd r = rk[i], b = bk ? bk[i] : r;
        const cd e = xs[i] - xk[i];
        x[2 * i] = cf{(float)(r.x * s), (float)(r.y * s)};
        x[2 * i + 1] = cf{(float)(b.x * s), (float)(b.y * s)};
        const cf ti = cf{(float)((e.x - b.x) * s), (float)((e.y - b.y) * s)};
        t[i] = ti;
        v = (double)ti.x * ti.x + (double)ti.y * ti.y;
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s2 += red[w];
        atomicAdd(scal + 2, s2);
    }
}

template <typename T>
bool galloc(T** p, size_t n)
{
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess;
}

size_t bwd_a_smem() { return sizeof(float) * (2 * GNN_W * (GNN_W + 1) + (size_t)GWARPS * 2 * GNN_W * GNN_W); }

}  // namespace

int gnn_setup(Gnn& G, int M, int ltri, int nx, int nnb, const int* nachbar)
{
    gnn_free(G);
    G.M = M;
    std::vector<int> nbr((size_t)M * GNN_D, -1), nsm((size_t)M * GNN_D, 0), rev((size_t)M * GNN_D, 0);
    auto put = [&](int i, int j, long long sidx) {
        for (int d = 0; d < GNN_D; ++d)
            if (nbr[(size_t)i * GNN_D + d] < 0) {
                nbr[(size_t)i * GNN_D + d] = j;
                nsm[(size_t)i * GNN_D + d] = (int)sidx;
                return true;
            }
        return false;
    };
    bool ok = true;
    if (ltri == 0) {
        for (int i = 0; i < M; ++i) {
            if (i > 0) ok &= put(i, i - 1, (long long)M + i - 1);
            if (i < M - 1) ok &= put(i, i + 1, (long long)M + i);
            if (i >= nx) ok &= put(i, i - nx, 2LL * M + i - nx);
            if (i < M - nx) ok &= put(i, i + nx, 2LL * M + i);
        }
    } else {
        for (int i = 0; i < M; ++i)
            for (int k = 0; k < nnb; ++k) {
                const int id = nachbar[(size_t)k * M + i];
                if (id > 0) ok &= put(i, id - 1, (long long)k * M + i);
            }
    }
    if (!ok) return CRT_ERR_UNSUPPORTED;
    // position of i in the list of each of its neighbours j (graph symmetric)
    for (int j = 0; j < M; ++j)
        for (int q = 0; q < GNN_D; ++q) {
            const int i = nbr[(size_t)j * GNN_D + q];
            if (i < 0) continue;
            int found = -1;
            for (int d = 0; d < GNN_D; ++d)
                if (nbr[(size_t)i * GNN_D + d] == j) found = d;
            if (found < 0) return CRT_ERR_UNSUPPORTED;   // not symmetric
            rev[(size_t)j * GNN_D + q] = found;
        }
    int nsm_count = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm_count, cudaDevAttrMultiProcessorCount, dev);
    G.nblk = std::max(1, nsm_count) * 4;
    const size_t MW = (size_t)M * GNN_W;
    bool a = galloc(&G.d_nbr, (size_t)M * GNN_D * 2) && galloc(&G.d_nsm, (size_t)M * GNN_D) &&
             galloc(&G.d_a, (size_t)M * GNN_D) && galloc(&G.d_w, GNN_NPARAM) && galloc(&G.d_wb, GNN_NPARAM) &&
             galloc(&G.d_m, GNN_NPARAM) && galloc(&G.d_v, GNN_NPARAM) && galloc(&G.d_g, GNN_NPARAM) &&
             galloc(&G.d_part, (size_t)G.nblk * GNN_NPARAM) && galloc(&G.d_h, (GNN_L + 1) * MW) &&
             galloc(&G.d_agg, GNN_L * MW) && galloc(&G.d_du, 2 * MW) && galloc(&G.d_x, (size_t)M * 4) &&
             galloc(&G.d_out, (size_t)M * 2) && galloc(&G.d_scal, 4);
    if (!a) {
        gnn_free(G);
        return CRT_ERR_ALLOC;
    }
    std::vector<int> nbr_rev(nbr);
    nbr_rev.insert(nbr_rev.end(), rev.begin(), rev.end());
    if (cudaMemcpy(G.d_nbr, nbr_rev.data(), nbr_rev.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(G.d_nsm, nsm.data(), nsm.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(G.d_w, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(G.d_wb, 0, GNN_NPARAM * sizeof(unsigned short)) != cudaSuccess ||
        cudaMemset(G.d_m, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(G.d_v, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(G.d_g, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess) {
        gnn_free(G);
        return CRT_ERR_CUDA;
    }
    G.ready = 1;
    return 0;
}

void gnn_free(Gnn& G)
{
    for (auto& r : G.recs) {
        cudaFree(r.x);
        cudaFree(r.t);
    }
    for (float* p : G.edge_sets) cudaFree(p);
    void* ptrs[] = {G.d_nbr, G.d_nsm, G.d_a, G.d_w, G.d_wb, G.d_m, G.d_v, G.d_g, G.d_part,
                    G.d_h, G.d_agg, G.d_du, G.d_x, G.d_out, G.d_scal};
    for (void* p : ptrs) cudaFree(p);
    G = Gnn{};
}

int gnn_init(Gnn& G, unsigned long long seed)
{
    // Glorot-uniform weights: U(-sqrt(6/(in+out)), +), from a seeded 64-bit
    // linear congruential generator (reproducible on every host).
    std::vector<float> w(GNN_NPARAM);
    unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto uni = [&]() {
        st = st * 6364136223846793005ULL + 1442695040888963407ULL;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int in, int out) {
        const double b = std::sqrt(6.0 / (in + out));
        for (int q = 0; q < in * out; ++q) w[off + q] = (float)((2.0 * uni() - 1.0) * b);
    };
    fill(GNN_OFF_IN, GNN_F, GNN_W);
    for (int l = 0; l < GNN_L; ++l) {
        fill(GNN_OFF_L + l * GNN_LSTRIDE, GNN_W, GNN_W);
        fill(GNN_OFF_L + l * GNN_LSTRIDE + GNN_W * GNN_W, GNN_W, GNN_W);
    }
    // a small output layer: the untrained correction starts near zero
    for (int q = 0; q < GNN_W * GNN_O; ++q) w[GNN_OFF_OUT + q] = (float)((2.0 * uni() - 1.0) * 1e-3);
    return gnn_set_weights(G, w.data());
}

int gnn_set_weights(Gnn& G, const float* w)
{
    if (cudaMemcpy(G.d_w, w, GNN_NPARAM * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(G.d_m, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(G.d_v, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(G.d_g, 0, GNN_NPARAM * sizeof(float)) != cudaSuccess)
        return CRT_ERR_CUDA;
    G.t_adam = 0;
    k_gnn_round<<<(GNN_NPARAM + 255) / 256, 256>>>(G.d_w, G.d_wb);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : CRT_ERR_CUDA;
}

void launch_gnn_edges(const Gnn& G, const double* cgfac, const double* smatm, double lam, cudaStream_t s)
{
    const int n = G.M * GNN_D;
    k_gnn_edges<<<(n + 255) / 256, 256, 0, s>>>(G.d_nbr, G.d_nsm, cgfac, smatm, lam, G.d_a, G.M);
}

static void forward(Gnn& G, const float* a, bool keep, const CGState* st, cudaStream_t s)
{
    const size_t MW = (size_t)G.M * GNN_W;
    k_gnn_in<<<G.nblk, GT, 0, s>>>(G.d_wb, G.d_x, G.d_h, G.M, st);
    for (int l = 0; l < GNN_L; ++l)
        k_gnn_layer<<<G.nblk, GT, 0, s>>>(G.d_wb, l, G.d_h + l * MW, G.d_h + (l + 1) * MW,
                                          keep ? G.d_agg + l * MW : nullptr, G.d_nbr, a, G.M, st);
}

void launch_gnn_apply(Gnn& G, const cd* r, const cd* zb, cd* z, const CGState* st, cudaStream_t s)
{
    k_gnn_norm<<<1, 1024, 0, s>>>(r, G.M, G.d_scal, st);
    k_gnn_feat<<<(G.M + 255) / 256, 256, 0, s>>>(r, zb, G.d_scal, G.d_x, G.M, st);
    forward(G, G.d_a, false, st, s);
    k_gnn_out_apply<<<G.nblk, GT, 0, s>>>(G.d_wb, G.d_h + (size_t)GNN_L * G.M * GNN_W, r, zb, G.d_scal, z, G.M, st);
}

void launch_gnn_record_grad(Gnn& G, const GnnRecordSet& R, float gscale, cudaStream_t s)
{
    const size_t MW = (size_t)G.M * GNN_W;
    const float* a = G.edge_sets[R.sys];
    k_gnn_feat_rec<<<(G.M + 255) / 256, 256, 0, s>>>(R.x, G.d_x, G.M);
    forward(G, a, true, nullptr, s);
    const float tinv = R.tnorm2 > 0.0f ? 1.0f / R.tnorm2 : 0.0f;
    float* du = G.d_du;
    float* dh = G.d_du + MW;
    k_gnn_out_loss<<<G.nblk, GT, sizeof(float) * GWARPS * GNN_W * GNN_O, s>>>(
        G.d_wb, G.d_h + GNN_L * MW, R.t, tinv, du, G.d_part, G.d_scal + 1, G.M);
    const size_t sa = bwd_a_smem();
    cudaFuncSetAttribute(k_gnn_bwd_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sa);
    for (int l = GNN_L - 1; l >= 0; --l) {
        // du holds du_l for the output of layer l (h_{l+1}); hp = h_l
        k_gnn_bwd_a<<<G.nblk, GT, sa, s>>>(G.d_wb, l, G.d_h + l * MW, G.d_agg + l * MW, du, dh, G.d_part, G.M);
        k_gnn_bwd_b<<<G.nblk, GT, 0, s>>>(G.d_h + l * MW, G.d_agg + l * MW, dh, G.d_nbr, G.d_nbr + (size_t)G.M * GNN_D,
                                          a, G.M);
        std::swap(du, dh);
    }
    k_gnn_bwd_in<<<G.nblk, GT, 0, s>>>(G.d_x, du, G.d_part, G.M);
    k_gnn_reduce<<<(GNN_NPARAM + 255) / 256, 256, 0, s>>>(G.d_part, G.nblk, gscale, G.d_g);
}

void launch_gnn_adam(Gnn& G, float lr, cudaStream_t s)
{
    ++G.t_adam;
    const float b1c = 1.0f - std::pow(0.9f, (float)G.t_adam), b2c = 1.0f - std::pow(0.999f, (float)G.t_adam);
    k_gnn_adam<<<(GNN_NPARAM + 255) / 256, 256, 0, s>>>(G.d_w, G.d_m, G.d_v, G.d_g, G.d_wb, lr, b1c, b2c);
}

void launch_gnn_round(Gnn& G, cudaStream_t s)
{
    k_gnn_round<<<(GNN_NPARAM + 255) / 256, 256, 0, s>>>(G.d_w, G.d_wb);
}

void launch_gnn_make_record(Gnn& G, GnnRecordSet& R, const cd* rk, const cd* bk, const cd* xk, const cd* xs,
                            cudaStream_t s)
{
    cudaMemsetAsync(G.d_scal + 2, 0, sizeof(double), s);
    k_gnn_norm<<<1, 1024, 0, s>>>(rk, G.M, G.d_scal, nullptr);
    k_gnn_make_rec<<<(G.M + 255) / 256, 256, 0, s>>>(rk, bk, xk, xs, G.d_scal, R.x, R.t, G.M);
}
