// hj_common.cuh -- shared definitions for the hegjoin_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "hegjoin_b200.h"
#include "hj_workspace.h"

namespace hj {

constexpr int kMaxK = 16;          // indexed dimensions supported
constexpr int kMaxD = 1024;        // dataset dimensions supported
constexpr uint32_t kSentinelKey = 0xFFFFFFFFu;

// ---- error handling --------------------------------------------------------
void set_error(const char* fmt, ...);
void count_launch();
uint64_t launch_count();
uint64_t thread_launch_count();   // launches made by the calling thread

#define HJ_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e__ = (call);                                                       \
        if (e__ != cudaSuccess) {                                                       \
            ::hj::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,                  \
                            cudaGetErrorString(e__));                                   \
            return e__ == cudaErrorMemoryAllocation ? HJ_ERR_OOM : HJ_ERR_CUDA;         \
        }                                                                               \
    } while (0)

#define HJ_TRY(...)                       \
    do {                                  \
        hj_status s__ = (__VA_ARGS__);    \
        if (s__ != HJ_OK) return s__;     \
    } while (0)

#define HJ_LAUNCHED()                                                                   \
    do {                                                                                \
        ::hj::count_launch();                                                           \
        cudaError_t e__ = cudaGetLastError();                                           \
        if (e__ != cudaSuccess) {                                                       \
            ::hj::set_error("%s:%d kernel launch: %s", __FILE__, __LINE__,              \
                            cudaGetErrorString(e__));                                   \
            return e__ == cudaErrorNoKernelImageForDevice ? HJ_ERR_NO_DEVICE : HJ_ERR_CUDA; \
        }                                                                               \
    } while (0)

// Status forms of HJ_CUDA / HJ_LAUNCHED for code that must release what it
// holds before returning (they record the error and return it instead).
inline hj_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return HJ_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? HJ_ERR_OOM : HJ_ERR_CUDA;
}
inline hj_status launch_status(const char* file, int line) {
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return HJ_OK;
    set_error("%s:%d kernel launch: %s", file, line, cudaGetErrorString(e));
    return e == cudaErrorNoKernelImageForDevice ? HJ_ERR_NO_DEVICE : HJ_ERR_CUDA;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- device buffers ----------------------------------------------------------
// Fault injection for tests (hj_debug_fail_alloc): while armed with n > 0, the
// n-th dalloc from then on fails the way an out-of-memory would.
bool injected_alloc_failure();   // hj_index.cu
bool injected_alloc_failure_armed();

// Stream-ordered device allocation; freed with dfree on the same stream.
template <typename T>
hj_status dalloc(T** p, size_t count, cudaStream_t st) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (injected_alloc_failure()) {
        set_error("device allocation of %zu bytes failed: injected failure", count * sizeof(T));
        return HJ_ERR_OOM;
    }
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), count * sizeof(T), st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        *p = nullptr;
        return HJ_ERR_OOM;
    }
    return HJ_OK;
}
template <typename T>
void dfree(T*& p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
}

// The device temporaries of one call: everything allocated through the guard is
// freed (in the order of its stream) when the guard goes out of scope, on every
// return path, unless it was handed over with keep() (pool blocks only: use
// alloc_pool for a buffer that will outlive the guard).
class Scratch {
  public:
    explicit Scratch(cudaStream_t st) : st_(st), ws_(current_workspace()) {
        if (ws_ && ws_->stream != st) ws_ = nullptr;
        if (ws_) {
            mark_ = ws_->top;
            depth_ = ++ws_->depth;
        }
    }
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    ~Scratch() {
        for (void* p : held_) cudaFreeAsync(p, st_);
        if (ws_) {
            ws_->top = mark_;
            --ws_->depth;
        }
    }
    template <typename T>
    hj_status alloc(T** p, size_t count) {
        if (ws_ && depth_ == ws_->depth && !injected_alloc_failure_armed()) {
            const size_t bytes = ((std::max<size_t>(count, 1) * sizeof(T)) + 255) & ~size_t(255);
            if (ws_->top + bytes <= ws_->cap) {
                *p = reinterpret_cast<T*>(ws_->base + ws_->top);
                ws_->top += bytes;
                return HJ_OK;
            }
        }
        return alloc_pool(p, count);
    }
    template <typename T>
    hj_status alloc_pool(T** p, size_t count) {
        hj_status s = dalloc(p, count, st_);
        if (s == HJ_OK) held_.push_back(*p);
        return s;
    }
    // Free one temporary now (a pool block goes back to the pool for the next
    // allocation; a workspace block is given back when the guard ends).
    template <typename T>
    void release(T*& p) {
        if (drop(p)) dfree(p, st_);
        p = nullptr;
    }
    // Hand a buffer to a longer-lived owner: the guard no longer frees it.
    template <typename T>
    T* keep(T* p) {
        drop(p);
        return p;
    }
    // Take charge of a buffer allocated elsewhere (freed with the others).
    template <typename T>
    T* adopt(T* p) {
        if (p) held_.push_back(p);
        return p;
    }

  private:
    bool drop(const void* p) {
        for (size_t i = 0; i < held_.size(); ++i)
            if (held_[i] == p) {
                held_[i] = held_.back();
                held_.pop_back();
                return true;
            }
        return false;
    }
    cudaStream_t st_;
    Workspace* ws_ = nullptr;
    size_t mark_ = 0;
    uint32_t depth_ = 0;
    std::vector<void*> held_;
};

// Raise a kernel's dynamic shared-memory limit once per (kernel, size), safe
// when several host threads launch joins concurrently.
hj_status ensure_smem_ptr(const void* kern, size_t bytes);   // hj_index.cu
template <typename K>
hj_status ensure_smem(K kern, size_t bytes) {
    return ensure_smem_ptr(reinterpret_cast<const void*>(kern), bytes);
}

inline int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

inline uint32_t bits_for(uint64_t max_value) {
    uint32_t b = 0;
    while (b < 64 && (max_value >> b) != 0) ++b;
    return b;
}

// ---- sort / scan primitives (hj_sort.cu) ---------------------------------------
// Exclusive scan of n u32 values into u64 (in and out may not alias).
hj_status scan_u32_to_u64(const uint32_t* in, uint64_t* out, uint64_t n, cudaStream_t st);
// In-place exclusive scan of u32 values (total must fit in u32).
hj_status scan_u32_inplace(uint32_t* data, uint64_t n, cudaStream_t st);
// In-place exclusive scan of doubles.
hj_status scan_f64_inplace(double* data, uint64_t n, cudaStream_t st);
// Stable LSD radix sort of (key, value) pairs on the low `nbits` key bits.
// On return the sorted data is in (keys, vals) (tmp buffers are scratch of n).
hj_status radix_sort_u64_u32(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                             uint64_t n, uint32_t nbits, cudaStream_t st);
hj_status radix_sort_u32_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                             uint64_t n, uint32_t nbits, cudaStream_t st);
// Sum of n u64 values (device result).
hj_status reduce_sum_u64(const uint64_t* in, uint64_t n, uint64_t* d_out, cudaStream_t st);

// ---- device helpers -------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Pair output buffer shared by the refine kernels.  Warps reserve CHUNK slots
// at a time from `cursor`; a reservation past `capacity` sets `overflow` and
// the batch is re-run by the host with smaller work.  Unused slots of the last
// chunk of every warp are filled with kSentinelKey keys.
struct PairSink {
    uint32_t* keys;
    uint32_t* vals;
    unsigned long long* cursor;
    unsigned long long capacity;
    uint32_t* overflow;
};

constexpr uint32_t kSinkChunk = 256;

// Per-warp reservation state, kept uniform across the warp.
struct WarpChunk {
    unsigned long long base;
    uint32_t used;
    uint32_t cap;   // 0 = none / overflowed
};

__device__ __forceinline__ void warp_chunk_init(WarpChunk& c) {
    c.base = 0;
    c.used = 0;
    c.cap = 0;
}

// Fill the unused tail of the warp's chunk with sentinels (call by the whole warp).
__device__ __forceinline__ void warp_chunk_close(const PairSink& s, WarpChunk& c) {
    if (c.cap == 0) return;
    for (uint32_t i = c.used + lane_id(); i < c.cap; i += 32) s.keys[c.base + i] = kSentinelKey;
    c.used = c.cap;
}

__device__ __forceinline__ bool warp_chunk_reserve(const PairSink& s, WarpChunk& c, uint32_t need) {
    // Called by the whole warp with a warp-uniform `need` (<= kSinkChunk).
    if (c.cap != 0 && c.used + need <= c.cap) return true;
    warp_chunk_close(s, c);
    unsigned long long base = 0;
    if (lane_id() == 0) base = atomicAdd(s.cursor, (unsigned long long)kSinkChunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base + kSinkChunk > s.capacity) {
        if (lane_id() == 0) atomicExch(s.overflow, 1u);
        c.cap = 0;
        c.used = 0;
        return false;
    }
    c.base = base;
    c.used = 0;
    c.cap = kSinkChunk;
    return true;
}

// Append, for every lane, `cnt` pairs: the lane's j-th pair is pair_of(j)
// (a uint2 of (key, value)).  Whole warp must call.  Returns false on overflow
// (pairs dropped; the batch will be re-run).
template <typename PairFn>
__device__ __forceinline__ bool warp_emit(const PairSink& s, WarpChunk& c, uint32_t cnt, PairFn&& pair_of) {
    // exclusive prefix of cnt across the warp
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane_id() >= (uint32_t)o) incl += t;
    }
    uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return true;
    uint32_t excl = incl - cnt;
    bool ok = true;
    uint32_t done = 0;  // pairs of the warp already written
    while (done < total) {
        uint32_t room = (c.cap != 0) ? c.cap - c.used : 0;
        if (room == 0) {
            if (!warp_chunk_reserve(s, c, 1)) { ok = false; break; }
            room = c.cap - c.used;
        }
        uint32_t take = min(room, total - done);
        // lane's pairs with warp-rank in [done, done + take)
        uint32_t lo = max(excl, done), hi = min(excl + cnt, done + take);
        for (uint32_t r = lo; r < hi; ++r) {
            unsigned long long pos = c.base + c.used + (r - done);
            uint2 kv = pair_of(r - excl);
            s.keys[pos] = kv.x;
            s.vals[pos] = kv.y;
        }
        c.used += take;
        done += take;
    }
    return ok;
}

// Append the pairs named by every lane's 32-bit hit mask, written out in
// coalesced runs: output slot i of the warp's hits is produced by lane i % 32,
// which finds the hit's owner lane (binary search over the inclusive prefix of
// the mask counts) and its bit (n-th set bit), then calls pair_of(owner, bit).
// Whole warp must call.  Returns false on overflow (pairs dropped; the batch
// will be re-run).
// With an owner value: every lane passes a value of its own (its row's id, say)
// and pair_of(owner, bit, value of the owner lane) receives the owner's, taken
// by a shuffle while the warp is converged.
template <typename PairFn>
__device__ __forceinline__ bool warp_emit_masks_v(const PairSink& s, WarpChunk& c, uint32_t mask, uint32_t val,
                                                  PairFn&& pair_of) {
    if (!__any_sync(0xffffffffu, mask != 0u)) return true;
    const uint32_t lane = lane_id();
    const uint32_t cnt = __popc(mask);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    bool ok = true;
    uint32_t done = 0;
    while (done < total) {
        uint32_t room = (c.cap != 0) ? c.cap - c.used : 0;
        if (room == 0) {
            if (!warp_chunk_reserve(s, c, 1)) { ok = false; break; }
            room = c.cap - c.used;
        }
        const uint32_t take = min(room, total - done);
        for (uint32_t b0 = 0; b0 < take; b0 += 32) {
            const uint32_t r = done + b0 + lane;   // the warp-wide rank this lane writes
            uint32_t owner = 0;                    // number of lanes whose inclusive count is <= r
#pragma unroll
            for (uint32_t st = 16; st > 0; st >>= 1) {
                const uint32_t inc = __shfl_sync(0xffffffffu, incl, owner + st - 1);
                if (inc <= r) owner += st;
            }
            owner = min(owner, 31u);
            const uint32_t o_incl = __shfl_sync(0xffffffffu, incl, owner);
            const uint32_t o_cnt = __shfl_sync(0xffffffffu, cnt, owner);
            const uint32_t o_mask = __shfl_sync(0xffffffffu, mask, owner);
            const uint32_t o_val = __shfl_sync(0xffffffffu, val, owner);
            const uint32_t k = r - (o_incl - o_cnt);                  // the owner's k-th hit (0-based)
            const uint32_t bit = __fns(o_mask, 0, (int)k + 1);       // 0xFFFFFFFF if there is none
            if (b0 + lane < take && bit < 32u) {
                const unsigned long long pos = c.base + c.used + b0 + lane;
                const uint2 kv = pair_of(owner, bit, o_val);
                s.keys[pos] = kv.x;
                s.vals[pos] = kv.y;
            }
        }
        c.used += take;
        done += take;
    }
    return ok;
}
template <typename PairFn>
__device__ __forceinline__ bool warp_emit_masks(const PairSink& s, WarpChunk& c, uint32_t mask, PairFn&& pair_of) {
    return warp_emit_masks_v(s, c, mask, 0u,
                             [&](uint32_t owner, uint32_t bit, uint32_t) { return pair_of(owner, bit); });
}

}  // namespace hj
