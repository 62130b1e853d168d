// hj_noalloc.cu -- grid geometry without any device allocation.
//
// hj_grid_geometry keeps its per-block partial minima/maxima in a buffer it
// allocates for each call.  Some callers cannot allocate device memory at the
// point where they need the geometry: a process that reserves all of its
// device memory up front (a serving process sized to its HBM budget, or one
// sharing the GPU under a fixed quota) and must never fail on an allocation
// later.  hj_grid_geometry_noalloc serves them: its scratch is the file-scope
// device array below, so a call allocates nothing.  The call copies the
// reduced minima/maxima to host memory and synchronises its stream, so it
// cannot run on a stream that is being captured into a CUDA graph.
//
// Limits and sharing: the array holds partials for at most kNaBlocks blocks x
// kNaMaxK indexed dimensions (k <= 16; any n below 2^32), 151,808 bytes,
// resident on every GPU that loads the library until the process exits.  All
// calls on a device share it and it keeps the last call's contents (every
// slot a call reads is written by that call first), so calls that overlap on
// the GPU (different streams, or host threads without ordering) race and must
// be serialised by the caller.  The first call on each device looks up the
// array's device address (cudaGetSymbolAddress) with that device current; the
// address is looked up again when the device's context has changed since (for
// example after cudaDeviceReset).
#include <algorithm>
#include <cmath>
#include <mutex>

#include <cuda.h>

#include "hj_internal.h"

namespace hj {
namespace {

constexpr uint32_t kNaBlocks = 592;   // 4 blocks per SM on 148 SMs
constexpr uint32_t kNaMaxK = 16;
constexpr uint32_t kNaScratch = 2 * kNaBlocks * kNaMaxK + 2 * kNaMaxK;   // doubles

// per-block partials [min | max][dim][block], then the reduced [min | max][dim]
static __device__ __align__(256) double g_na_scratch[kNaScratch];

std::mutex g_na_mu;
double* g_na_addr[64] = {};
CUcontext g_na_ctx[64] = {};   // the context each cached address belongs to

// cuCtxGetCurrent through the runtime's driver entry-point query (the library
// does not link libcuda directly).
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<Fn>(p);
        return static_cast<Fn>(nullptr);
    }();
    CUcontext c = nullptr;
    if (fn) fn(&c);
    return c;
}

template <typename T>
__global__ void k_na_minmax(const T* __restrict__ db, uint32_t n, uint32_t d, uint32_t k, double* __restrict__ sc) {
    __shared__ T smin[kNaMaxK][8], smax[kNaMaxK][8];
    const uint32_t w = threadIdx.x >> 5;
    for (uint32_t j = 0; j < k; ++j) {
        T mn = db[j], mx = db[j];
        // 64-bit index: a 32-bit one would wrap past n near 2^32 and never end the loop
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (uint64_t)gridDim.x * blockDim.x) {
            T v = db[i * d + j];
            mn = v < mn ? v : mn;
            mx = v > mx ? v : mx;
        }
        for (int o = 16; o > 0; o >>= 1) {
            T a = __shfl_down_sync(0xffffffffu, mn, o), b = __shfl_down_sync(0xffffffffu, mx, o);
            mn = a < mn ? a : mn;
            mx = b > mx ? b : mx;
        }
        if ((threadIdx.x & 31u) == 0) { smin[j][w] = mn; smax[j][w] = mx; }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        T mn = smin[j][0], mx = smax[j][0];
        for (uint32_t x = 1; x < (blockDim.x >> 5); ++x) {
            mn = smin[j][x] < mn ? smin[j][x] : mn;
            mx = smax[j][x] > mx ? smax[j][x] : mx;
        }
        sc[(size_t)j * gridDim.x + blockIdx.x] = (double)mn;
        sc[(size_t)(kNaMaxK + j) * gridDim.x + blockIdx.x] = (double)mx;
    }
}

__global__ void k_na_final(double* __restrict__ sc, uint32_t nblocks, uint32_t k) {
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        double mn = sc[(size_t)j * nblocks], mx = sc[(size_t)(kNaMaxK + j) * nblocks];
        for (uint32_t b = 1; b < nblocks; ++b) {
            mn = fmin(mn, sc[(size_t)j * nblocks + b]);
            mx = fmax(mx, sc[(size_t)(kNaMaxK + j) * nblocks + b]);
        }
        sc[2 * kNaBlocks * kNaMaxK + j] = mn;
        sc[2 * kNaBlocks * kNaMaxK + kNaMaxK + j] = mx;
    }
}

template <typename T>
hj_status na_geometry(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, double* h_min, double* h_max,
                      uint32_t* h_nc, uint64_t* h_total, double* sc, cudaStream_t st) {
    const uint32_t nblocks = std::min<uint32_t>(kNaBlocks, std::max<uint32_t>(1, (n + 255) / 256));
    k_na_minmax<T><<<nblocks, 256, 0, st>>>(db, n, d, k, sc);
    HJ_LAUNCHED();
    k_na_final<<<1, 32, 0, st>>>(sc, nblocks, k);
    HJ_LAUNCHED();
    double mm[2 * kNaMaxK];   // host stack: no allocation
    HJ_CUDA(cudaMemcpyAsync(mm, sc + 2 * kNaBlocks * kNaMaxK, sizeof(mm), cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    uint64_t total = 1;
    for (uint32_t j = 0; j < k; ++j) {
        // the same arithmetic as generateNDGridDimensions (main.cu:489-509), in T
        T mnA = (T)mm[j] - eps;
        T mxA = (T)mm[kNaMaxK + j] + eps;
        T r = (mxA - mnA) / eps;
        uint32_t nc = (uint32_t)std::ceil(r);
        if (h_min) h_min[j] = (double)mnA;
        if (h_max) h_max[j] = (double)mxA;
        if (h_nc) h_nc[j] = nc;
        total *= nc;
    }
    if (h_total) *h_total = total;
    return HJ_OK;
}

}  // namespace
}  // namespace hj

using namespace hj;

extern "C" hj_status hj_grid_geometry_noalloc(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype,
                                              double eps, double* h_min_arr, double* h_max_arr, uint32_t* h_n_cells,
                                              uint64_t* h_total_cells, void* stream) {
    if (!d_db || n == 0 || d == 0 || k == 0 || k > d || !(eps > 0) || (dtype != HJ_F32 && dtype != HJ_F64)) {
        set_error("hj_grid_geometry_noalloc: invalid arguments (n=%u d=%u k=%u eps=%g)", n, d, k, eps);
        return HJ_ERR_INVALID;
    }
    if (k > kNaMaxK) {
        set_error("hj_grid_geometry_noalloc: k=%u indexed dimensions exceed the static scratch's maximum of %u", k,
                  kNaMaxK);
        return HJ_ERR_INVALID;
    }
    int dev = 0;
    HJ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("hj_grid_geometry_noalloc: device %d out of range", dev);
        return HJ_ERR_INVALID;
    }
    double* sc = nullptr;
    {
        // the device's current context (cudaGetDevice above made it current)
        const CUcontext ctx = current_context();
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_addr[dev] || g_na_ctx[dev] != ctx) {
            // first call on this device: the array's device address (host code cannot use its name)
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
            if (e != cudaSuccess) {
                set_error("hj_grid_geometry_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return e == cudaErrorNoKernelImageForDevice ? HJ_ERR_NO_DEVICE : HJ_ERR_CUDA;
            }
            g_na_addr[dev] = static_cast<double*>(p);
            g_na_ctx[dev] = ctx;
        }
        sc = g_na_addr[dev];
    }
    cudaStream_t st = as_stream(stream);
    if (dtype == HJ_F32)
        return na_geometry<float>((const float*)d_db, n, d, k, (float)eps, h_min_arr, h_max_arr, h_n_cells,
                                  h_total_cells, sc, st);
    return na_geometry<double>((const double*)d_db, n, d, k, eps, h_min_arr, h_max_arr, h_n_cells, h_total_cells, sc,
                               st);
}
