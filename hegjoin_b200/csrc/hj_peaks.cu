// hj_peaks.cu -- measured peaks of the pipes the refine kernels run on.
//
// The roofline denominators the benchmark reports beside the driver-measured
// copy bandwidth and cuBLAS bf16 rate: this library's own kernels, timed with
// CUDA events on the caller's stream.
//   * FP32 FMA: chains of fma.rn.f32, and of the packed fma.rn.f32x2 the exact
//     refine uses (two FMAs per lane and instruction);
//   * FP64 FMA: chains of fma.rn.f64 (the FP64 exact refine);
//   * tensor core, kind::f16: M = 128 x N = 256 x K = 16 MMAs from shared memory
//     into TMEM, back to back from two issuing threads with one accumulator each
//     (the refine's issue pattern), FP16 and BF16 inputs, FP32 accumulation.
// Each kernel runs one CTA shape over every SM for long enough (tens of ms)
// that launch costs vanish; a flop is one multiply or one add.
#include <cudaTypedefs.h>

#include <algorithm>

#include "hj_internal.h"
#include "hj_tc.cuh"

namespace hj {
namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_peak_ffma(float* out, int iters, float b, float c) {
    float a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __fmaf_rn(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 1234.5f) out[0] = s;   // keeps the chains; never true for these inputs
}

__global__ void __launch_bounds__(256) k_peak_ffma2(float* out, int iters, float b, float c) {
    unsigned long long a[kChains];
    const unsigned long long bb = ((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(b);
    const unsigned long long cc = ((unsigned long long)__float_as_uint(c) << 32) | __float_as_uint(c);
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        const float x = threadIdx.x * 1e-3f + k;
        a[k] = ((unsigned long long)__float_as_uint(x + 0.5f) << 32) | __float_as_uint(x);
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[k]) : "l"(bb), "l"(cc));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += __uint_as_float((uint32_t)a[k]) + __uint_as_float((uint32_t)(a[k] >> 32));
    if (s == 1234.5f) out[0] = s;
}

__global__ void __launch_bounds__(256) k_peak_dfma(double* out, int iters, double b, double c) {
    double a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3 + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __fma_rn(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 1234.5) out[0] = s;
}

constexpr uint32_t kPeakA = 128 * 64;   // A: 128 rows of one 32-element K block (64 bytes, 64-byte swizzle)
constexpr uint32_t kPeakB = 256 * 64;   // B: 256 rows

// Two issuing threads (warp 0 and warp 1, lane 0), each `iters` MMAs into its own
// 256-column accumulator, then one commit each; every thread waits (bounded) for
// both commits before the TMEM is released.  Operand contents do not matter.
__global__ void __launch_bounds__(128, 1) k_peak_mma(uint32_t idesc, int iters, uint32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t base = tc::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    uint8_t* a_t = smem;
    uint8_t* b_t = smem + kPeakA;
    uint64_t* bar = reinterpret_cast<uint64_t*>(b_t + kPeakB);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    uint32_t* abortp = tslot + 1;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    for (uint32_t i = tid; i < (kPeakA + kPeakB) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(smem)[i] = 0u;
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        *abortp = 0;
        tc::fence_mbar_init();
    }
    tc::fence_proxy_async_smem();   // the zeroed operands, written by ordinary stores, are read by the tensor core
    if (warp == 1) {
        tc::tmem_alloc(tslot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    if (warp < 2 && lane == 0) {
        const uint32_t acc = tmem + warp * 256u;
        const uint32_t a_base = tc::smem_u32(a_t), b_base = tc::smem_u32(b_t);
        for (int i = 0; i < iters; ++i) {
            const uint32_t kin = (uint32_t)(i & 1) * 32u;
            tc::mma_f16(acc, tc::desc_kmajor_sw64(a_base + kin), tc::desc_kmajor_sw64(b_base + kin), idesc,
                        i > 0 ? 1u : 0u);
        }
        tc::mma_commit(&bar[warp]);
    }
    __syncwarp();
    tc::mbar_wait(&bar[0], 0, abortp, err, 4000000000ll);
    tc::mbar_wait(&bar[1], 0, abortp, err, 4000000000ll);
    tc::fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

template <typename K>
hj_status time_launch(K&& launch, cudaStream_t st, float* ms) {
    cudaEvent_t e0, e1;
    HJ_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_status(cudaGetLastError(), "cudaEventCreate");
    }
    hj_status s = launch();   // warm-up
    if (s == HJ_OK) s = cuda_status(cudaEventRecord(e0, st), "record");
    if (s == HJ_OK) s = launch();
    if (s == HJ_OK) s = cuda_status(cudaEventRecord(e1, st), "record");
    if (s == HJ_OK) s = cuda_status(cudaEventSynchronize(e1), "sync");
    if (s == HJ_OK) s = cuda_status(cudaEventElapsedTime(ms, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

}  // namespace
}  // namespace hj

using namespace hj;

extern "C" hj_status hj_measure_peaks(hj_peaks* out, void* stream) {
    if (!out) { set_error("hj_measure_peaks: null argument"); return HJ_ERR_INVALID; }
    *out = hj_peaks{};
    cudaStream_t st = as_stream(stream);
    Scratch tmp(st);
    double* sink = nullptr;
    uint32_t* err = nullptr;
    HJ_TRY(tmp.alloc(&sink, 1));
    HJ_TRY(tmp.alloc(&err, 1));
    HJ_CUDA(cudaMemsetAsync(err, 0, 4, st));
    const int sms = num_sms();
    const unsigned blocks = (unsigned)sms * 8;   // 2048 threads per SM
    const double threads = (double)blocks * 256;
    float ms = 0;
    {
        const int iters = 100000;
        HJ_TRY(time_launch([&] {
            k_peak_ffma<<<blocks, 256, 0, st>>>(reinterpret_cast<float*>(sink), iters, 1.0000001f, 1e-7f);
            return launch_status(__FILE__, __LINE__);
        }, st, &ms));
        out->fp32_fma_tflops = 2.0 * kChains * iters * threads / (ms * 1e-3) / 1e12;
        HJ_TRY(time_launch([&] {
            k_peak_ffma2<<<blocks, 256, 0, st>>>(reinterpret_cast<float*>(sink), iters, 1.0000001f, 1e-7f);
            return launch_status(__FILE__, __LINE__);
        }, st, &ms));
        out->fp32x2_fma_tflops = 4.0 * kChains * iters * threads / (ms * 1e-3) / 1e12;
        const int diters = 20000;
        HJ_TRY(time_launch([&] {
            k_peak_dfma<<<blocks, 256, 0, st>>>(sink, diters, 1.0000001, 1e-7);
            return launch_status(__FILE__, __LINE__);
        }, st, &ms));
        out->fp64_fma_tflops = 2.0 * kChains * diters * threads / (ms * 1e-3) / 1e12;
    }
    {
        const int iters = 100000;
        const size_t smem = 1024 + kPeakA + kPeakB + 64;
        HJ_TRY(ensure_smem(k_peak_mma, std::max<size_t>(smem, 116 * 1024)));   // one CTA per SM
        const size_t dyn = std::max<size_t>(smem, 116 * 1024);
        for (int bf = 0; bf < 2; ++bf) {
            const uint32_t idesc = tc::idesc_f16((uint32_t)bf, 128, 256);
            HJ_TRY(time_launch([&] {
                k_peak_mma<<<sms, 128, dyn, st>>>(idesc, iters, err);
                return launch_status(__FILE__, __LINE__);
            }, st, &ms));
            const double tf = 2.0 * 128 * 256 * 16 * 2.0 * iters * sms / (ms * 1e-3) / 1e12;
            if (bf) out->bf16_mma_tflops = tf; else out->f16_mma_tflops = tf;
        }
    }
    uint32_t herr = 0;
    HJ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("hj_measure_peaks: a bounded wait expired"); return HJ_ERR_TIMEOUT; }
    return HJ_OK;
}
