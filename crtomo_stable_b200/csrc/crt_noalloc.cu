// crt_noalloc.cu -- crt_voltages_noalloc: the four-pole voltages (rtrafo at
// the electrode nodes + bvolti / bvolt) for callers that cannot allocate
// device memory.
//
// Who needs it: code that owns all of its device memory up front and may
// not call cudaMalloc / cudaFree from the point where it evaluates
// voltages -- for example an application whose device memory comes from its
// own pool or framework allocator, or a real-time acquisition loop that
// forbids allocation (and the implicit synchronisation it brings) after
// start-up.  Such a caller passes device buffers for every input and
// output; the intermediate table of electrode-node potentials that the
// context-based path (crt_forward) keeps in its own allocation lives here
// in a file-scope __device__ array instead.
//
// The array holds at most CRT_NOALLOC_MAX_EANZ x CRT_NOALLOC_MAX_EANZ
// complex values (512 x 512 x 16 B = 4 MiB); every GPU that loads the library
// keeps it until the process exits.  All calls share it: calls that overlap
// on the GPU (different streams, or host threads without ordering) race on
// its contents.  The only part that must start at zero, the status word, is
// cleared at the start of every call; the potential table is fully
// rewritten by every call before it is read.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/crt_b200.h"
#include "crt_common.cuh"

#define CRT_NOALLOC_MAX_EANZ 512
#define CRT_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) cd g_noalloc_hel[CRT_NOALLOC_MAX_EANZ * CRT_NOALLOC_MAX_EANZ];
static __device__ __align__(256) int g_noalloc_status[64];

namespace {

struct NoallocSymbols {
    cd* hel = nullptr;
    int* status = nullptr;
};

std::mutex g_noalloc_mutex;
NoallocSymbols g_noalloc_sym[CRT_NOALLOC_MAX_DEVICES];
bool g_noalloc_ready[CRT_NOALLOC_MAX_DEVICES] = {};

// Device addresses of the scratch arrays for the current device, looked up
// once per device (the host-side names are stand-ins, not device addresses).
int noalloc_symbols(NoallocSymbols* out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= CRT_NOALLOC_MAX_DEVICES) return CRT_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ready[dev]) {
        NoallocSymbols s;
        cudaError_t e1 = cudaGetSymbolAddress((void**)&s.hel, g_noalloc_hel);
        cudaError_t e2 = cudaGetSymbolAddress((void**)&s.status, g_noalloc_status);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            std::fprintf(stderr, "crt_voltages_noalloc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            return CRT_ERR_CUDA;
        }
        g_noalloc_sym[dev] = s;
        g_noalloc_ready[dev] = true;
    }
    *out = g_noalloc_sym[dev];
    return CRT_OK;
}

// hel[c*L + p] = sum_k kwnwi(k) kpot(enr(p), c, k) / pi (enr 1-based)
__global__ void k_noalloc_hel(const cd* __restrict__ kpot, const double* __restrict__ kwnwi,
                              const int32_t* __restrict__ enr, int n, int L, int K, int swrtr, double pi,
                              cd* __restrict__ hel, int* status)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L * L) return;
    const int p = t % L, c = t / L;
    const int node = enr[p] - 1;
    if (node < 0 || node >= n) {   // electrode node outside the mesh (errnr 29)
        atomicMax(status, 29);
        hel[(size_t)c * L + p] = cd{0.0, 0.0};
        return;
    }
    cd s{0.0, 0.0};
    if (swrtr == 0) {
        s = kpot[(size_t)c * n + node];
    } else {
        for (int k = 0; k < K; ++k) s += kpot[((size_t)k * L + c) * n + node] * kwnwi[k];
        s = s / pi;
    }
    hel[(size_t)c * L + p] = s;
}

__device__ __forceinline__ cd noalloc_term(const cd* hel, int L, int ep, int ec)
{
    const double f = (double)(min(ep, 1) * min(ec, 1));
    return hel[(size_t)(max(ec, 1) - 1) * L + (max(ep, 1) - 1)] * f;
}

__global__ void k_noalloc_volt(const cd* __restrict__ hel, const int32_t* __restrict__ strnr,
                               const int32_t* __restrict__ vnr, const double* __restrict__ kfak, int L, int N,
                               int ldc, int mode, cd* __restrict__ volt, cd* __restrict__ sigmaa, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int s = strnr[i], v = vnr[i];
    const int e1 = s % 10000, e2 = (s - e1) / 10000, e3 = v % 10000, e4 = (v - e3) / 10000;
    if (min(min(e1, e2), min(e3, e4)) < 0 || max(max(e1, e2), max(e3, e4)) > L) {
        atomicMax(status, 46);
        volt[i] = cd{0.0, 0.0};
        sigmaa[i] = cd{0.0, 0.0};
        return;
    }
    cd d1 = noalloc_term(hel, L, e4, e2), d2 = noalloc_term(hel, L, e4, e1);
    cd d3 = noalloc_term(hel, L, e3, e2), d4 = noalloc_term(hel, L, e3, e1);
    cd vt = (d1 - d2) - (d3 - d4);
    if (ldc) vt = cd{vt.x, 0.0};
    volt[i] = vt;
    if (mode == 0) {
        const double m = hypot(vt.x, vt.y);
        if (m == 0.0) {
            atomicMax(status, (int)CRT_ERR_ZERO_VOLT);
            sigmaa[i] = cd{0.0, 0.0};
        } else {
            sigmaa[i] = cd{-log(m), -atan2(vt.y, vt.x)};
        }
    } else {
        sigmaa[i] = vt * (kfak ? kfak[i] : 1.0);
    }
}

}  // namespace

extern "C" int32_t crt_voltages_noalloc(const double* kpot, const double* kwnwi, const int32_t* enr,
                                        const int32_t* strnr, const int32_t* vnr, int32_t sanz, int32_t eanz,
                                        int32_t kwnanz, int32_t nanz, int32_t swrtr, int32_t ldc, int32_t mode,
                                        const double* kfak, double* volt, double* sigmaa, void* stream)
{
    if (!kpot || !kwnwi || !enr || !strnr || !vnr || !volt || !sigmaa || sanz <= 0 || eanz <= 0 || kwnanz <= 0 ||
        nanz < 0 || (mode != 0 && mode != 1))
        return CRT_ERR_ARG;
    if (eanz > CRT_NOALLOC_MAX_EANZ) {
        std::fprintf(stderr,
                     "crt_voltages_noalloc: eanz = %d exceeds the %d electrodes its static scratch holds; "
                     "use crt_forward instead\n",
                     (int)eanz, CRT_NOALLOC_MAX_EANZ);
        return CRT_ERR_ARG;
    }
    // an error left pending by earlier, unrelated work is reported as such
    // (and left in place for its owner) rather than charged to this call
    if (cudaError_t pre = cudaPeekAtLastError(); pre != cudaSuccess) {
        std::fprintf(stderr, "crt_voltages_noalloc: a CUDA error was pending before the call: %s\n",
                     cudaGetErrorString(pre));
        return CRT_ERR_CUDA;
    }
    NoallocSymbols sym;
    if (int e = noalloc_symbols(&sym)) return e;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(sym.status, 0, sizeof(int), st) != cudaSuccess) return CRT_ERR_CUDA;
    if (nanz == 0) return cudaStreamSynchronize(st) == cudaSuccess ? CRT_OK : CRT_ERR_CUDA;
    const int nel = eanz * eanz;
    k_noalloc_hel<<<(nel + 255) / 256, 256, 0, st>>>(reinterpret_cast<const cd*>(kpot), kwnwi, enr, sanz, eanz, kwnanz,
                                                     swrtr, std::acos(-1.0), sym.hel, sym.status);
    k_noalloc_volt<<<(nanz + 255) / 256, 256, 0, st>>>(sym.hel, strnr, vnr, kfak, eanz, nanz, ldc, mode,
                                                       reinterpret_cast<cd*>(volt), reinterpret_cast<cd*>(sigmaa),
                                                       sym.status);
    // nothing was pending on entry, so a launch error seen here is this call's
    if (cudaGetLastError() != cudaSuccess) return CRT_ERR_CUDA;
    int status = 0;
    if (cudaMemcpyAsync(&status, sym.status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CRT_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CRT_ERR_CUDA;
    return status;
}
