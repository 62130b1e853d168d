// hj_sort.cu -- device scan and stable LSD radix sort.
//
// Replaces the Thrust sort / sort_by_key / unique calls of the reference
// (GPU.cu:249-251, GPU.cu:285, GPU.cu:1543).  The radix sort is a
// reduce-then-scan LSD sort with 8-bit digits: per pass a tile histogram
// kernel, an exclusive scan of the (digit-major) histogram table and a stable
// scatter that ranks each tile's keys in shared memory.  Only the low `nbits`
// key bits are sorted, so a 21-bit point-id key costs three passes.

#include "hj_common.cuh"

namespace hj {
namespace {

constexpr int kScanBlock = 1024;
constexpr int kScanItems = 8;               // per thread
constexpr int kScanTile = kScanBlock * kScanItems;

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;                // keys per thread per tile
constexpr int kRsTile = kRsThreads * kRsItems;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRadix = 256;

// ---- scan --------------------------------------------------------------------
template <typename In, typename Out>
__global__ void k_tile_sums(const In* __restrict__ in, uint64_t n, Out* __restrict__ sums) {
    __shared__ Out warp_tot[kScanBlock / 32];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    Out acc = 0;
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kScanBlock + threadIdx.x;
        if (idx < n) acc += (Out)in[idx];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane_id() == 0) warp_tot[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        Out v = warp_tot[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = v;
    }
}

// Exclusive scan of `sums` (m entries) in place by one block.
template <typename Out>
__global__ void k_scan_sums(Out* sums, uint64_t m) {
    __shared__ Out part[kScanBlock];
    uint64_t per = (m + kScanBlock - 1) / kScanBlock;
    uint64_t b = threadIdx.x * per, e = min(m, b + per);
    Out acc = 0;
    for (uint64_t i = b; i < e; ++i) acc += sums[i];
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        Out t = (threadIdx.x >= (unsigned)o) ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += t;
        __syncthreads();
    }
    Out run = part[threadIdx.x] - acc;
    for (uint64_t i = b; i < e; ++i) {
        Out v = sums[i];
        sums[i] = run;
        run += v;
    }
}

// Block-wide exclusive scan of one tile plus the tile's offset (none when
// offsets is null: a scan of a single tile).  Every element is read and
// written by the same thread, so the scan may run in place.
template <typename In, typename Out>
__global__ void k_scan_tiles(const In* in, Out* out, uint64_t n, const Out* __restrict__ offsets) {
    __shared__ Out warp_tot[kScanBlock / 32];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    Out v[kScanItems];
    Out acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + i;
        v[i] = idx < n ? (Out)in[idx] : 0;
        acc += v[i];
    }
    // warp inclusive scan of per-thread totals
    Out incl = acc;
    for (int o = 1; o < 32; o <<= 1) {
        Out t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane_id() >= (uint32_t)o) incl += t;
    }
    if (lane_id() == 31) warp_tot[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        Out w = warp_tot[threadIdx.x];
        Out wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            Out t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane_id() >= (uint32_t)o) wi += t;
        }
        warp_tot[threadIdx.x] = wi - w;
    }
    __syncthreads();
    Out run = (offsets ? offsets[blockIdx.x] : Out(0)) + warp_tot[threadIdx.x >> 5] + incl - acc;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] = run;
        run += v[i];
    }
}

template <typename In, typename Out>
hj_status exclusive_scan(const In* in, Out* out, uint64_t n, cudaStream_t st) {
    if (n == 0) return HJ_OK;
    uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        // one tile: a single launch and no partial sums (small scans are most of a
        // small join's, including every pass of the radix sorts of small inputs)
        k_scan_tiles<In, Out><<<1, kScanBlock, 0, st>>>(in, out, n, nullptr);
        HJ_LAUNCHED();
        return HJ_OK;
    }
    Scratch tmp(st);
    Out* sums = nullptr;
    HJ_TRY(tmp.alloc(&sums, tiles));
    k_tile_sums<In, Out><<<(unsigned)tiles, kScanBlock, 0, st>>>(in, n, sums);
    HJ_LAUNCHED();
    k_scan_sums<Out><<<1, kScanBlock, 0, st>>>(sums, tiles);
    HJ_LAUNCHED();
    k_scan_tiles<In, Out><<<(unsigned)tiles, kScanBlock, 0, st>>>(in, out, n, sums);
    HJ_LAUNCHED();
    return HJ_OK;
}

// ---- radix sort ----------------------------------------------------------------
template <typename K>
__global__ void k_rs_hist(const K* __restrict__ keys, uint64_t n, uint32_t shift, uint32_t* __restrict__ hist,
                          uint32_t ntiles) {
    __shared__ uint32_t h[kRsWarps][kRadix];
    for (int i = threadIdx.x; i < kRsWarps * kRadix; i += kRsThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    uint32_t w = threadIdx.x >> 5;
    for (int i = 0; i < kRsItems; ++i) {
        uint64_t idx = base + (uint64_t)i * kRsThreads + threadIdx.x;
        if (idx < n) atomicAdd(&h[w][(uint32_t)(keys[idx] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int dgt = threadIdx.x; dgt < kRadix; dgt += kRsThreads) {
        uint32_t s = 0;
        for (int j = 0; j < kRsWarps; ++j) s += h[j][dgt];
        hist[(uint64_t)dgt * ntiles + blockIdx.x] = s;
    }
}

// Stable scatter: tile elements are visited in order (round r covers tile
// positions [r*256, r*256+256)), ranked by (earlier rounds, earlier warps,
// earlier lanes) among keys with the same digit.
template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const K* __restrict__ keys, const uint32_t* __restrict__ vals,
                                                           K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                           uint64_t n, uint32_t shift, const uint32_t* __restrict__ offs,
                                                           uint32_t ntiles) {
    __shared__ uint32_t run[kRadix];           // running count per digit (tile-global offset)
    __shared__ uint32_t wcnt[kRsWarps][kRadix + 1];
    for (int dgt = threadIdx.x; dgt < kRadix; dgt += kRsThreads) run[dgt] = offs[(uint64_t)dgt * ntiles + blockIdx.x];
    for (int i = threadIdx.x; i < kRsWarps * (kRadix + 1); i += kRsThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    for (int r = 0; r < kRsItems; ++r) {
        uint64_t idx = base + (uint64_t)r * kRsThreads + threadIdx.x;
        bool valid = idx < n;
        K key = valid ? keys[idx] : K(0);
        uint32_t val = valid ? vals[idx] : 0u;
        uint32_t dgt = valid ? ((uint32_t)(key >> shift) & 0xFFu) : (uint32_t)kRadix;
        uint32_t peers = __match_any_sync(0xffffffffu, dgt);
        uint32_t rank = __popc(peers & lanemask_lt());
        uint32_t leader = __ffs(peers) - 1;
        if (lane == leader) wcnt[w][dgt] = __popc(peers);
        __syncthreads();
        // per digit: exclusive prefix across warps, then advance the running count
        for (int dd = threadIdx.x; dd < kRadix; dd += kRsThreads) {
            uint32_t acc = run[dd];
            for (int j = 0; j < kRsWarps; ++j) {
                uint32_t c = wcnt[j][dd];
                wcnt[j][dd] = acc;
                acc += c;
            }
            run[dd] = acc;
        }
        __syncthreads();
        if (valid) {
            uint32_t dst = wcnt[w][dgt] + rank;
            keys_out[dst] = key;
            vals_out[dst] = val;
        }
        __syncthreads();
        // every digit slot now holds a prefix value; reset the table for the next round
        for (int j = threadIdx.x; j < kRsWarps * (kRadix + 1); j += kRsThreads) (&wcnt[0][0])[j] = 0;
        __syncthreads();
    }
}

template <typename K>
hj_status radix_sort(K* keys, uint32_t* vals, K* keys_tmp, uint32_t* vals_tmp, uint64_t n, uint32_t nbits,
                     cudaStream_t st) {
    if (n <= 1 || nbits == 0) return HJ_OK;
    if (n >= (1ull << 32)) {
        set_error("radix sort: %llu elements exceed 2^32", (unsigned long long)n);
        return HJ_ERR_INVALID;
    }
    uint32_t ntiles = (uint32_t)((n + kRsTile - 1) / kRsTile);
    Scratch tmp(st);
    uint32_t* hist = nullptr;
    HJ_TRY(tmp.alloc(&hist, (size_t)kRadix * ntiles));
    K* src_k = keys; uint32_t* src_v = vals;
    K* dst_k = keys_tmp; uint32_t* dst_v = vals_tmp;
    uint32_t passes = (nbits + 7) / 8;
    for (uint32_t p = 0; p < passes; ++p) {
        uint32_t shift = p * 8;
        k_rs_hist<K><<<ntiles, kRsThreads, 0, st>>>(src_k, n, shift, hist, ntiles);
        HJ_LAUNCHED();
        HJ_TRY(exclusive_scan<uint32_t, uint32_t>(hist, hist, (uint64_t)kRadix * ntiles, st));
        k_rs_scatter<K><<<ntiles, kRsThreads, 0, st>>>(src_k, src_v, dst_k, dst_v, n, shift, hist, ntiles);
        HJ_LAUNCHED();
        std::swap(src_k, dst_k);
        std::swap(src_v, dst_v);
    }
    if (src_k != keys) {
        HJ_CUDA(cudaMemcpyAsync(keys, src_k, n * sizeof(K), cudaMemcpyDeviceToDevice, st));
        HJ_CUDA(cudaMemcpyAsync(vals, src_v, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    }
    return HJ_OK;
}

__global__ void k_reduce_u64(const uint64_t* __restrict__ in, uint64_t n, unsigned long long* out) {
    unsigned long long acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += in[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane_id() == 0 && acc) atomicAdd(out, acc);
}

}  // namespace

hj_status scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, cudaStream_t st) {
    return exclusive_scan<uint32_t, uint64_t>(in, out, n, st);
}
hj_status scan_u32_inplace(uint32_t* data, uint64_t n, cudaStream_t st) {
    return exclusive_scan<uint32_t, uint32_t>(data, data, n, st);
}
hj_status scan_f64_inplace(double* data, uint64_t n, cudaStream_t st) {
    return exclusive_scan<double, double>(data, data, n, st);
}
hj_status radix_sort_u64_u32(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, uint64_t n,
                             uint32_t nbits, cudaStream_t st) {
    return radix_sort<uint64_t>(keys, vals, keys_tmp, vals_tmp, n, nbits, st);
}
hj_status radix_sort_u32_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp, uint64_t n,
                             uint32_t nbits, cudaStream_t st) {
    return radix_sort<uint32_t>(keys, vals, keys_tmp, vals_tmp, n, nbits, st);
}
hj_status reduce_sum_u64(const uint64_t* in, uint64_t n, uint64_t* d_out, cudaStream_t st) {
    HJ_CUDA(cudaMemsetAsync(d_out, 0, sizeof(uint64_t), st));
    if (n == 0) return HJ_OK;
    unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)num_sms() * 8);
    k_reduce_u64<<<grid, 256, 0, st>>>(in, n, reinterpret_cast<unsigned long long*>(d_out));
    HJ_LAUNCHED();
    return HJ_OK;
}

}  // namespace hj
