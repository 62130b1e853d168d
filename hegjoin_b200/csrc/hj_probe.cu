// hj_probe.cu -- arithmetic probe for the reference's distance expression.
//
// kernel.cu:350-353 accumulates
//     runningTotalDist += (database[...] - point[l]) * (database[...] - point[l]);
// and the reference builds it with nvcc's defaults (makefile:10: -O3, no
// --fmad flag, so --fmad=true).  This kernel compiles that expression verbatim
// with the same defaults, so its bits show whether nvcc contracts it to
// fma(diff, diff, acc).  The refine kernels of this library never rely on the
// compiler for that choice: they call __fmaf_rn / __fma_rn explicitly.

#include "hj_internal.h"

namespace hj {
namespace {
template <typename T>
__global__ void k_probe_sqdist(const T* a, const T* b, uint32_t n, uint32_t d, T* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T runningTotalDist = 0;
    for (uint32_t l = 0; l < d; ++l) {
        runningTotalDist += (a[(size_t)i * d + l] - b[(size_t)i * d + l]) * (a[(size_t)i * d + l] - b[(size_t)i * d + l]);
    }
    out[i] = runningTotalDist;
}
}  // namespace
}  // namespace hj

extern "C" hj_status hj_probe_sqdist(const void* d_a, const void* d_b, uint32_t n, uint32_t d, int dtype, void* d_out,
                                     void* stream) {
    using namespace hj;
    if (!d_a || !d_b || !d_out || n == 0 || d == 0) { set_error("hj_probe_sqdist: invalid arguments"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    if (dtype == HJ_F32)
        k_probe_sqdist<float><<<(n + 255) / 256, 256, 0, st>>>((const float*)d_a, (const float*)d_b, n, d, (float*)d_out);
    else
        k_probe_sqdist<double><<<(n + 255) / 256, 256, 0, st>>>((const double*)d_a, (const double*)d_b, n, d, (double*)d_out);
    HJ_LAUNCHED();
    return HJ_OK;
}
