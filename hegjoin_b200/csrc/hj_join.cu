// hj_join.cu -- batch estimator, batched join driver and device result table.
//
// Reference counterparts:
//   GPUBatchEst_v2                          GPU.cu:403-779
//   distanceTableNDGridBatches              GPU.cu:787-1702
//   constructNeighborTableKeyValueWithPtrs  GPU.cu:1731-1776
//
// B200 design.  The reference samples every 10th query, refines it, sizes a
// 50M-pair buffer from max-of-adjacent-sample extrapolation, and then runs
// batches on three streams, each followed by a Thrust key sort, a PCIe copy of
// all pairs and a host table build.  Here:
//   * the estimator refines every s-th work item (cell block) in count-only
//     mode and extrapolates per item with the max of the two adjacent samples
//     (the reference's rule, GPU.cu:608-633), in the workload order;
//   * one pair buffer sized from the estimate and from free HBM holds a whole
//     batch; batches are cut at half the buffer (the reference allocates twice
//     its nominal buffer, GPU.cu:1042-1062) and a batch whose pairs overflow
//     the buffer is split in two and re-run, instead of writing out of bounds;
//   * pairs are grouped by query id on the device with the library's radix
//     sort, and the neighbour table (the device form of neighborTableLookup,
//     structs.h:35-41) is built on the device; nothing crosses PCIe unless the
//     caller exports it.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <queue>
#include <sstream>

#include "hj_internal.h"

namespace hj {
uint32_t plain_query_block(int dtype);
bool plain_counts_queries(const hj_index* ix);
hj_status launch_refine_plain(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                              const PairSink& sink, uint32_t count_only, unsigned long long* block_counts,
                              uint32_t* qcount, cudaStream_t st);
hj_status tc_prepare(hj_index* ix, int kind, cudaStream_t st);
uint32_t tc_query_block();
hj_status launch_refine_tc(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                           const PairSink& sink, const PairSink& band, uint32_t count_only,
                           unsigned long long* block_counts, unsigned long long* stats, uint32_t* err,
                           cudaStream_t st);
hj_status launch_band_recheck(const hj_index* ix, const uint32_t* bq, const uint32_t* bc,
                              const unsigned long long* band_used, unsigned long long band_cap,
                              const PairSink& sink, uint32_t nblocks, cudaStream_t st);
uint64_t plain_emit_warps(uint32_t nblocks);
uint64_t tc_emit_warps(uint32_t nblocks);
double tc_delta(const hj_index* ix);
double tc_band_ratio(const hj_index* ix);
bool tc_supported(const hj_index* ix, int kind);
int tc_get_epi(const hj_index* ix);
void tc_set_epi(hj_index* ix, int epi);
void tc_set_defer(hj_index* ix, bool defer);
}  // namespace hj

struct hj_result {
    uint32_t n = 0;
    cudaStream_t stream = nullptr;       // the join's stream; buffers are freed in its order
    std::vector<uint32_t*> vals;
    std::vector<uint32_t*> keys;
    std::vector<uint64_t> counts;
    uint32_t** d_batch_vals = nullptr;   // device array of the per-batch value pointers
    hj_nt_entry* table = nullptr;        // n entries
    uint64_t total = 0;
};

namespace hj {
namespace {

__global__ void k_pick_samples(const HjBlock* __restrict__ blocks, uint32_t nblocks, uint32_t stride,
                               uint32_t nsamp, HjBlock* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsamp) return;
    out[i] = blocks[min(nblocks - 1, i * stride)];
}

// Estimated pairs per work item, on the device: the sampled rate (pairs per
// query) of the item's sample group, or the larger of its group's and the next
// group's for items between samples, times the item's queries
// (GPUBatchEst_v2's extrapolation, GPU.cu:608-633, on work items); est[nblocks]
// = 0 for the exclusive scan.  Queries x candidates of every item add up in *cand.
__global__ void k_item_estimates(const HjBlock* __restrict__ blocks, uint32_t nblocks, uint32_t stride,
                                 uint32_t nsamp, const HjBlock* __restrict__ sblocks,
                                 const unsigned long long* __restrict__ scnt, double* __restrict__ est,
                                 double* __restrict__ cand) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double c = 0;
    if (i < nblocks) {
        const uint32_t s = min(i / stride, nsamp - 1);
        auto rate = [&](uint32_t q) { return (double)scnt[q] / (double)max(1u, sblocks[q].q1 - sblocks[q].q0); };
        double r = rate(s);
        if (i % stride != 0) r = fmax(r, rate(min(nsamp - 1, s + 1)));
        const HjBlock b = blocks[i];
        est[i] = r * (double)(b.q1 - b.q0);
        c = (double)b.nb * (double)(b.q1 - b.q0);
    } else if (i == nblocks) {
        est[i] = 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if (lane_id() == 0 && c > 0) atomicAdd(cand, c);
}

// Batch cuts: item i > 0 starts a batch where the exclusive prefix of the
// estimates crosses a multiple of the budget, so a batch's estimate stays below
// the budget plus its last item's.
__global__ void k_batch_cuts(const double* __restrict__ pre, uint32_t nblocks, double budget,
                             uint32_t* __restrict__ cuts, unsigned int* __restrict__ ncuts) {
    const uint32_t i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nblocks) return;
    if (floor(pre[i] / budget) != floor(pre[i - 1] / budget)) cuts[atomicAdd(ncuts, 1u)] = i;
}

// Light work items (at most kLightCandidates candidates per query) go in cell
// order.  The workload order runs the heavy items first, which keeps the
// persistent refine balanced, but it scatters the many light items of sparse
// data over the whole grid: spatial neighbours, which read the same candidate
// cells and probe the same hash slots, then run far apart and miss in L2.  In
// cell (linear id) order consecutive light items share most of their stencil.
constexpr uint32_t kLightCandidates = 4096;
// Only lists this long are reordered: a small join saves the host round trip.
constexpr uint32_t kLightMinItems = 65536;

// Items whose cells have more candidates than `lim`: a prefix, since the items
// follow the workload order (candidates non-increasing).
__global__ void k_count_heavy(const HjBlock* __restrict__ b, uint32_t n, uint32_t lim, unsigned int* cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t heavy = __popc(__ballot_sync(0xffffffffu, i < n && b[i].nb > lim));
    if (lane_id() == 0 && heavy) atomicAdd(cnt, heavy);
}
__global__ void k_item_cells(const HjBlock* __restrict__ b, uint32_t m, uint32_t* __restrict__ cell,
                             uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    cell[i] = b[i].cell;
    idx[i] = i;
}
__global__ void k_gather_items(const HjBlock* __restrict__ in, const uint32_t* __restrict__ idx, uint32_t m,
                               HjBlock* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = in[idx[i]];
}

// Counters and flags of one join, in one device allocation.
struct JoinCtl {
    unsigned long long cursor;        // pair sink cursor of the current batch
    unsigned long long valid;         // pairs left after grouping (sentinels dropped)
    unsigned long long tc_acc;        // tensor-core filter: pairs accepted outside the band (this batch)
    unsigned long long tc_band;       // tensor-core filter: band pairs (this batch)
    unsigned long long band_cursor;   // band sink cursor of the current batch
    uint32_t head;                    // work-item queue head of the current launch
    uint32_t overflow;                // a sink ran out of room
    uint32_t timeout;                 // a bounded device-side wait expired
    uint32_t pad_;
};

// Start of a batch: both sink cursors, the overflow flag, the queue head and the
// filter's counters (the host adds up those of the batches that did not overflow).
__global__ void k_batch_reset(JoinCtl* c) {
    if (threadIdx.x == 0) {
        c->cursor = 0;
        c->band_cursor = 0;
        c->valid = 0;
        c->overflow = 0;
        c->head = 0;
        c->tc_acc = 0;
        c->tc_band = 0;
    }
}

// Grouping a batch's pairs by query id: a counting sort.  Keys are query ids
// below n (sentinel slots are skipped), so one pass counts the pairs per query,
// an exclusive scan over the n + 1 counters gives every query's first slot, and
// one more pass scatters each pair to its query's run.  Within a query the order
// of its pairs is not defined, as in the reference (whose key sort is unstable).
//
// Both passes work on tiles of 4,096 consecutive pairs per block.  A tile comes
// mostly from one or two work items, so it holds a few dozen distinct queries:
// the block gathers them in a shared-memory table (key -> slot, open addressing;
// lanes of a warp with the same key share one table operation) and issues one
// global atomic per query per tile instead of one per query per warp.  Keys
// that find the table full take their global atomics directly.
constexpr uint32_t kGrpPer = 16;                       // pairs per thread per tile
constexpr uint32_t kGrpTile = 256 * kGrpPer;           // pairs per block-tile
constexpr uint32_t kGrpSlots = 1024;                   // table slots (power of two)
constexpr uint32_t kGrpFull = 0xFFFFFFFFu;

// Slot of `key` in the block's table (inserting it), or kGrpFull.
__device__ __forceinline__ uint32_t grp_slot(uint32_t* hk, uint32_t key) {
    uint32_t h = (uint32_t)mix64(key) & (kGrpSlots - 1);
    for (uint32_t probe = 0; probe < 64; ++probe) {
        const uint32_t prev = atomicCAS(&hk[h], kSentinelKey, key);
        if (prev == kSentinelKey || prev == key) return h;
        h = (h + 1) & (kGrpSlots - 1);
    }
    return kGrpFull;
}

__global__ void __launch_bounds__(256) k_group_count(const uint32_t* __restrict__ keys, unsigned long long m,
                                                      uint32_t* __restrict__ cnt) {
    __shared__ uint32_t hk[kGrpSlots], hc[kGrpSlots];
    for (unsigned long long base = (unsigned long long)blockIdx.x * kGrpTile; base < m;
         base += (unsigned long long)gridDim.x * kGrpTile) {
        for (uint32_t s = threadIdx.x; s < kGrpSlots; s += blockDim.x) { hk[s] = kSentinelKey; hc[s] = 0; }
        __syncthreads();
#pragma unroll 4
        for (uint32_t j = 0; j < kGrpPer; ++j) {
            const unsigned long long i = base + j * 256ull + threadIdx.x;
            const uint32_t key = i < m ? keys[i] : kSentinelKey;
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            if (key != kSentinelKey && lane_id() == (uint32_t)(__ffs(peers) - 1)) {
                const uint32_t sl = grp_slot(hk, key);
                if (sl == kGrpFull) atomicAdd(&cnt[key], __popc(peers));
                else atomicAdd(&hc[sl], __popc(peers));
            }
        }
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < kGrpSlots; s += blockDim.x)
            if (hk[s] != kSentinelKey) atomicAdd(&cnt[hk[s]], hc[s]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_group_scatter(const uint32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vals, unsigned long long m,
                                                        uint32_t* __restrict__ cursor, uint32_t* __restrict__ keys_out,
                                                        uint32_t* __restrict__ vals_out) {
    __shared__ uint32_t hk[kGrpSlots], hc[kGrpSlots];
    for (unsigned long long base = (unsigned long long)blockIdx.x * kGrpTile; base < m;
         base += (unsigned long long)gridDim.x * kGrpTile) {
        for (uint32_t s = threadIdx.x; s < kGrpSlots; s += blockDim.x) { hk[s] = kSentinelKey; hc[s] = 0; }
        __syncthreads();
        // pass 1: the tile's pairs per query (the thread keeps its keys and values)
        uint32_t kk[kGrpPer], vv[kGrpPer];
#pragma unroll
        for (uint32_t j = 0; j < kGrpPer; ++j) {
            const unsigned long long i = base + j * 256ull + threadIdx.x;
            kk[j] = i < m ? keys[i] : kSentinelKey;
            vv[j] = i < m ? vals[i] : 0u;
        }
#pragma unroll
        for (uint32_t j = 0; j < kGrpPer; ++j) {
            const uint32_t key = kk[j];
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            if (key != kSentinelKey && lane_id() == (uint32_t)(__ffs(peers) - 1)) {
                const uint32_t sl = grp_slot(hk, key);
                if (sl != kGrpFull) atomicAdd(&hc[sl], __popc(peers));
            }
        }
        __syncthreads();
        // one global reservation per query of the tile; the slot's count becomes its cursor
        for (uint32_t s = threadIdx.x; s < kGrpSlots; s += blockDim.x)
            if (hk[s] != kSentinelKey) hc[s] = atomicAdd(&cursor[hk[s]], hc[s]);
        __syncthreads();
        // pass 2: place the pairs
#pragma unroll
        for (uint32_t j = 0; j < kGrpPer; ++j) {
            const uint32_t key = kk[j];
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            const uint32_t leader = __ffs(peers) - 1;
            uint32_t first = 0;
            if (key != kSentinelKey && lane_id() == leader) {
                uint32_t sl = kGrpFull;
                // the key is in the table unless the table was full when it came
                uint32_t h = (uint32_t)mix64(key) & (kGrpSlots - 1);
                for (uint32_t probe = 0; probe < 64; ++probe) {
                    const uint32_t k2 = hk[h];
                    if (k2 == key) { sl = h; break; }
                    if (k2 == kSentinelKey) break;
                    h = (h + 1) & (kGrpSlots - 1);
                }
                first = sl != kGrpFull ? atomicAdd(&hc[sl], __popc(peers)) : atomicAdd(&cursor[key], __popc(peers));
            }
            first = __shfl_sync(0xffffffffu, first, leader);
            if (key != kSentinelKey) {
                const uint32_t pos = first + __popc(peers & lanemask_lt());
                keys_out[pos] = key;
                vals_out[pos] = vv[j];
            }
        }
        __syncthreads();
    }
}

// constructNeighborTableKeyValueWithPtrs (GPU.cu:1731-1776) on the device, from
// the grouping's cursors: after the scatter, run_end[q] is one past query q's last
// pair in the batch's grouped arrays and its run starts at run_end[q - 1] (0 for
// q = 0), so every query with pairs gets its entry without a pass over the pairs.
__global__ void k_table_runs(const uint32_t* __restrict__ run_end, uint32_t n, uint32_t batch,
                             hj_nt_entry* __restrict__ table) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const uint32_t start = q ? run_end[q - 1] : 0u;
    const uint32_t end = run_end[q];
    if (end > start) table[q] = hj_nt_entry{batch, end - start, start};
}

__global__ void k_table_counts(const hj_nt_entry* __restrict__ t, uint32_t n, uint32_t* __restrict__ cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cnt[i] = t[i].count;
}

__global__ void k_csr_copy(const hj_nt_entry* __restrict__ t, uint32_t* const* __restrict__ bv, uint32_t n,
                           const uint64_t* __restrict__ off, uint32_t* __restrict__ out) {
    uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= n) return;
    hj_nt_entry e = t[q];
    if (!e.count) return;
    const uint32_t* src = bv[e.batch] + e.start;
    uint64_t o = off[q];
    for (uint32_t i = lane_id(); i < e.count; i += 32) out[o + i] = src[i];
}

__global__ void k_csr_keys(const hj_nt_entry* __restrict__ t, const uint32_t* __restrict__ vals, uint32_t n,
                           const uint64_t* __restrict__ off, uint64_t* __restrict__ keys64) {
    uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= n) return;
    uint32_t c = t[q].count;
    uint64_t o = off[q];
    for (uint32_t i = lane_id(); i < c; i += 32) keys64[o + i] = ((uint64_t)q << 32) | vals[o + i];
}

__global__ void k_unpack_vals(const uint64_t* __restrict__ keys64, uint64_t n, uint32_t* __restrict__ vals) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) vals[i] = (uint32_t)keys64[i];
}

__global__ void k_digest(const hj_nt_entry* __restrict__ t, uint32_t* const* __restrict__ bv, uint32_t n,
                         uint32_t* __restrict__ cnt, uint64_t* __restrict__ sum, uint64_t* __restrict__ xr) {
    uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (q >= n) return;
    hj_nt_entry e = t[q];
    uint64_t s = 0, x = 0;
    if (e.count) {
        const uint32_t* src = bv[e.batch] + e.start;
        for (uint32_t i = lane_id(); i < e.count; i += 32) {
            uint32_t v = src[i];
            s += mix64(v);
            x ^= mix64((uint64_t)v ^ 0x5bd1e9955bd1e995ull);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        x ^= __shfl_down_sync(0xffffffffu, x, o);
    }
    if (lane_id() == 0) {
        if (cnt) cnt[q] = e.count;
        if (sum) sum[q] = s;
        if (xr) xr[q] = x;
    }
}

struct Batch {
    uint32_t b0, b1;
};

// ---- autotuner ------------------------------------------------------------------------
// Tile-shape choices are timed once per (refine kind, d, dtype) on the
// estimator's count-only sample and remembered for the process; with
// HJ_TUNE_FILE set they are also read from / appended to that file
// ("kind d dtype choice" per line).  HJ_TUNE=0 disables timing (defaults used).
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

std::string tune_key(int kind, uint32_t d, int dtype) {
    std::ostringstream o;
    o << kind << ' ' << d << ' ' << dtype;
    return o.str();
}

bool tune_lookup(const std::string& key, int* choice) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (!g_tune_loaded) {
        g_tune_loaded = true;
        if (const char* f = std::getenv("HJ_TUNE_FILE")) {
            std::ifstream in(f);
            int k, c;
            uint32_t d;
            int dt;
            while (in >> k >> d >> dt >> c) g_tune[tune_key(k, d, dt)] = c;
        }
    }
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    *choice = it->second;
    return true;
}

void tune_store(const std::string& key, int choice) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = choice;
    if (const char* f = std::getenv("HJ_TUNE_FILE")) {
        std::ofstream out(f, std::ios::app);
        out << key << ' ' << choice << '\n';
    }
}

bool tuning_enabled() {
    const char* e = std::getenv("HJ_TUNE");
    return !(e && e[0] == '0');
}

// Tensor-core epilogue: with fewer than ~3% of its 32 x 32 chunks holding a hit, one vote
// per accumulator and a re-read of the hit chunks beats a vote per chunk (measured at
// d = 18 with 1.6% and at d = 90 with 6.4%).  HJ_TC_DEFER=0/1 forces either form (tests).
bool defer_for(double pairs, double cand) {
    if (const char* e = std::getenv("HJ_TC_DEFER")) return e[0] == '1';
    return cand > 0 && pairs * 1024.0 < 0.03 * cand;
}

float ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace hj

namespace hj {
// Re-associate a result with another stream for its frees.  The server calls
// this with the legacy default stream once a worker has synchronised its own
// stream, so results outlive the worker streams that produced them.
void result_set_stream(hj_result* r, cudaStream_t s) {
    if (r) r->stream = s;
}

namespace {

__global__ void k_pick_list(const HjBlock* __restrict__ blocks, const uint32_t* __restrict__ items, uint32_t m,
                            HjBlock* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = blocks[items[i]];
}

// Per-query digests of a grouped batch (keys ascending): (count, sum of
// mix64(id), xor of mix64(id ^ salt)) per query, added into (cnt, sum, xr).  A
// warp stages a walk of 512 consecutive pairs in shared memory (coalesced loads)
// and every lane folds its 16 consecutive ones serially.  Runs that begin and
// end inside a lane go out with one atomic triple.  A lane's last run may go on
// in the next lanes: a segmented scan over the lanes' last runs (equal keys
// chain; a lane whose last run continues the previous lane's holds one key
// only) gives each run's total up to every lane; the lane where the run ends
// writes it, or, when the next lane's first run continues it and that lane
// holds more runs, that lane adds its first run and writes it.  Long runs (a
// query with thousands of neighbours) cost one scan and a few atomics per 512
// pairs; a run crossing two walks is written by both (the digest adds up).
constexpr uint32_t kDigestPer = 16;                  // pairs per lane per walk
constexpr uint32_t kDigestSpan = 32 * kDigestPer;    // pairs per warp per walk
__device__ __forceinline__ void digest_out(uint32_t* cnt, unsigned long long* sum, unsigned long long* xr,
                                           uint32_t key, uint32_t c, unsigned long long s, unsigned long long x) {
    atomicAdd(&cnt[key], c);
    atomicAdd(&sum[key], s);
    atomicXor(&xr[key], x);
}
__global__ void __launch_bounds__(256) k_digest_accumulate(const uint32_t* __restrict__ keys,
                                                            const uint32_t* __restrict__ vals, unsigned long long n,
                                                            uint32_t* __restrict__ cnt, unsigned long long* __restrict__ sum,
                                                            unsigned long long* __restrict__ xr) {
    // per warp: the walk's keys and values, 16 per lane with one word of padding per lane
    // so that the lanes' serial reads fall in different banks
    __shared__ uint32_t sk[8][32 * (kDigestPer + 1)], sv[8][32 * (kDigestPer + 1)];
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const unsigned long long warps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long base = (((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kDigestSpan;
         base < n; base += warps * kDigestSpan) {
#pragma unroll
        for (uint32_t j = 0; j < kDigestPer; ++j) {
            const uint32_t e = j * 32 + lane;                          // element of the walk
            const uint32_t slot = (e / kDigestPer) * (kDigestPer + 1) + e % kDigestPer;
            const unsigned long long i = base + e;
            sk[w][slot] = i < n ? keys[i] : kSentinelKey;
            sv[w][slot] = i < n ? vals[i] : 0u;
        }
        __syncwarp();
        const uint32_t* mk = &sk[w][lane * (kDigestPer + 1)];
        const uint32_t* mv = &sv[w][lane * (kDigestPer + 1)];
        uint32_t fk = kSentinelKey, fc = 0, lk = mk[0], lc = 0;
        unsigned long long fs = 0, fx = 0, ls = 0, lx = 0;
        bool single = true;
#pragma unroll 4
        for (uint32_t j = 0; j < kDigestPer; ++j) {
            const uint32_t key = mk[j];
            if (key == kSentinelKey) break;   // sentinels only trail
            if (key != lk) {
                if (single) { fk = lk; fc = lc; fs = ls; fx = lx; single = false; }
                else digest_out(cnt, sum, xr, lk, lc, ls, lx);
                lk = key; lc = 0; ls = 0; lx = 0;
            }
            const uint32_t v = mv[j];
            lc += 1;
            ls += mix64(v);
            lx ^= mix64((uint64_t)v ^ 0x5bd1e9955bd1e995ull);
        }
        const uint32_t key_first = single ? lk : fk;
        // segmented scan of the last runs over the lanes
        unsigned long long s = ls, x = lx;
        uint32_t c = lc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t k2 = __shfl_up_sync(0xffffffffu, lk, o);
            const unsigned long long s2 = __shfl_up_sync(0xffffffffu, s, o);
            const unsigned long long x2 = __shfl_up_sync(0xffffffffu, x, o);
            const uint32_t c2 = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= (uint32_t)o && k2 == lk) { s += s2; x ^= x2; c += c2; }
        }
        const uint32_t pk = __shfl_up_sync(0xffffffffu, lk, 1);
        const unsigned long long ps = __shfl_up_sync(0xffffffffu, s, 1), px = __shfl_up_sync(0xffffffffu, x, 1);
        const uint32_t pc = __shfl_up_sync(0xffffffffu, c, 1);
        const uint32_t nk = __shfl_down_sync(0xffffffffu, key_first, 1);
        if (!single) {
            // the first run: complete here, joined with the previous lanes' run when it goes on from there
            if (lane > 0 && pk == fk) digest_out(cnt, sum, xr, fk, fc + pc, fs + ps, fx ^ px);
            else digest_out(cnt, sum, xr, fk, fc, fs, fx);
        }
        // the last run (with its earlier lanes) ends here unless the next lane goes on with it
        if (lk != kSentinelKey && (lane == 31 || nk != lk)) digest_out(cnt, sum, xr, lk, c, s, x);
        __syncwarp();
    }
}

// Timing events are taken from a per-thread pool and returned to it: creating and
// destroying them per launch is a driver call each, which concurrent joins (the
// serving loop's workers) would serialise on.
struct EventPool {
    std::vector<cudaEvent_t> free;
    ~EventPool() {
        for (cudaEvent_t e : free) cudaEventDestroy(e);
    }
};
thread_local EventPool t_events;

hj_status event_acquire(cudaEvent_t* e) {
    if (!t_events.free.empty()) {
        *e = t_events.free.back();
        t_events.free.pop_back();
        return HJ_OK;
    }
    return cuda_status(cudaEventCreate(e), "cudaEventCreate");
}

// CUDA events of the refine launches, returned to the pool on every return path.
struct EventPairs {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    ~EventPairs() {
        for (auto& e : ev) {
            if (e.first) t_events.free.push_back(e.first);
            if (e.second) t_events.free.push_back(e.second);
        }
    }
};

// What a join does with each grouped batch.
struct BatchHandler {
    virtual ~BatchHandler() = default;
    // `count` pairs of batch `batch`: query ids (ascending) in keys, neighbour ids
    // grouped by query in vals.  Both live in the join's reusable buffers and stay
    // valid in the order of `st` until the next batch's refine is enqueued.  With
    // pairs, run_end (n entries, in the order of `st` until the next batch's grouping)
    // holds one past each query's last pair: query q's run is
    // [run_end[q - 1] (0 for q = 0), run_end[q]).
    virtual hj_status on_batch(uint32_t batch, const uint32_t* keys, const uint32_t* vals, uint64_t count,
                               const uint32_t* run_end, cudaStream_t st) = 0;
    // Whether the handler can use two alternating sets of grouped arrays, and the event
    // (if any) after which the last batch's set may be reused.
    virtual bool can_overlap() const { return false; }
    virtual cudaEvent_t take_release() { return nullptr; }
};

// The batched join (distanceTableNDGridBatches, GPU.cu:787-1702): refine kind,
// work items (optionally this rank's share), estimator, result-buffer sizing,
// batches with overflow split-and-retry, grouping by query id.  Every device
// temporary lives in `tmp` and is freed on every return path.
// kept_bytes_per_pair: device bytes the handler keeps per result pair (left free);
// fixed_kept_bytes: what the caller already holds for the result (counted against
// opts.device_bytes_cap).
hj_status join_impl(hj_index* ix, const hj_join_opts* opts_in, cudaStream_t st, BatchHandler& handler,
                    double kept_bytes_per_pair, uint64_t fixed_kept_bytes, hj_join_stats* stats) {
    auto t_start = std::chrono::steady_clock::now();
    hj_join_opts opts;
    if (opts_in) opts = *opts_in; else hj_join_opts_default(&opts);
    if (opts.sample_rate <= 0 || opts.sample_rate > 1) opts.sample_rate = 0.02;
    if (opts.mem_fraction <= 0 || opts.mem_fraction > 0.95) opts.mem_fraction = 0.6;
    if (opts.shard_count > 1 && opts.shard_index >= opts.shard_count) {
        set_error("hj_join: shard_index %u out of range for %u shards", opts.shard_index, opts.shard_count);
        return HJ_ERR_INVALID;
    }
    Scratch tmp(st);
    uint64_t launches0 = thread_launch_count();
    hj_join_stats S{};
    HJ_TRY(hj_sort_by_workload(ix, st, nullptr));

    // ---- refine kind
    int refine = opts.refine;
    const bool auto_kind = refine == HJ_REFINE_AUTO;
    if (auto_kind)
        refine = (ix->dtype == HJ_F32 && ix->d >= 16 && tc_supported(ix, HJ_REFINE_TC_F16)) ? HJ_REFINE_TC_F16
                                                                                            : HJ_REFINE_EXACT;
    bool tc = refine == HJ_REFINE_TC_F16 || refine == HJ_REFINE_TC_BF16;
    if (tc) {
        if (!tc_supported(ix, refine)) {
            set_error("hj_join: the tensor-core filter needs float data with 8 <= d <= 188 and k <= 6");
            return HJ_ERR_UNSUPPORTED;
        }
        const hj_status ps = tc_prepare(ix, refine, st);
        if (ps != HJ_OK && !(auto_kind && ps == HJ_ERR_UNSUPPORTED)) return ps;
        // auto: data the filter cannot take (non-finite coordinates), or whose guard band is
        // wider than half the threshold (the filter would decide little), go to the exact path
        if (auto_kind && (ps != HJ_OK || tc_band_ratio(ix) > 0.5)) {
            refine = HJ_REFINE_EXACT;
            tc = false;
        }
        if (tc) S.filter_delta = tc_delta(ix);
    }
    S.refine_used = (uint32_t)refine;
    // the tile shape of each refine kernel fixes its work-item size
    const uint32_t qb = tc ? tc_query_block() : plain_query_block(ix->dtype);

    HjBlock* blocks = nullptr;
    uint32_t nblocks = 0;
    HJ_TRY(build_blocks(ix, qb, &blocks, &nblocks, st));
    tmp.adopt(blocks);
    if (!tc && nblocks >= kLightMinItems) {
        // the light items' tail in cell order (kLightCandidates)
        unsigned int* dh = nullptr;
        HJ_TRY(tmp.alloc(&dh, 1));
        HJ_CUDA(cudaMemsetAsync(dh, 0, sizeof(unsigned int), st));
        k_count_heavy<<<(nblocks + 255) / 256, 256, 0, st>>>(blocks, nblocks, kLightCandidates, dh);
        HJ_LAUNCHED();
        unsigned int heavy = 0;
        HJ_CUDA(cudaMemcpyAsync(&heavy, dh, sizeof(heavy), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        tmp.release(dh);
        const uint32_t m = nblocks - heavy;
        if (m > 1) {
            uint32_t *cell = nullptr, *idx = nullptr, *cell_t = nullptr, *idx_t = nullptr;
            HjBlock* out = nullptr;
            HJ_TRY(tmp.alloc(&cell, m));
            HJ_TRY(tmp.alloc(&idx, m));
            HJ_TRY(tmp.alloc(&cell_t, m));
            HJ_TRY(tmp.alloc(&idx_t, m));
            HJ_TRY(tmp.alloc(&out, m));
            k_item_cells<<<(m + 255) / 256, 256, 0, st>>>(blocks + heavy, m, cell, idx);
            HJ_LAUNCHED();
            HJ_TRY(radix_sort_u32_u32(cell, idx, cell_t, idx_t, m, bits_for(ix->nC), st));
            k_gather_items<<<(m + 255) / 256, 256, 0, st>>>(blocks + heavy, idx, m, out);
            HJ_LAUNCHED();
            HJ_CUDA(cudaMemcpyAsync(blocks + heavy, out, (size_t)m * sizeof(HjBlock), cudaMemcpyDeviceToDevice, st));
            tmp.release(out);
            tmp.release(idx_t);
            tmp.release(cell_t);
            tmp.release(idx);
            tmp.release(cell);
        }
    }
    if (opts.shard_count > 1) {
        // the item list on the host, for the costs of the share
        std::vector<HjBlock> hblocks(nblocks);
        if (nblocks) {
            HJ_CUDA(cudaMemcpyAsync(hblocks.data(), blocks, (size_t)nblocks * sizeof(HjBlock), cudaMemcpyDeviceToHost,
                                    st));
            HJ_CUDA(cudaStreamSynchronize(st));
        }
        // this rank's share of the items: greedy LPT on (candidates x queries) per item
        std::vector<uint64_t> cost(nblocks);
        for (uint32_t i = 0; i < nblocks; ++i) cost[i] = (uint64_t)hblocks[i].nb * (hblocks[i].q1 - hblocks[i].q0);
        std::vector<uint32_t> mine(std::max<uint32_t>(nblocks, 1));
        uint32_t n_mine = 0;
        HJ_TRY(hj_shard_plan_lpt(cost.data(), nblocks, opts.shard_count, opts.shard_index, mine.data(), &n_mine));
        uint32_t* d_items = nullptr;
        HjBlock* sel = nullptr;
        HJ_TRY(tmp.alloc(&d_items, std::max<uint32_t>(n_mine, 1)));
        HJ_TRY(tmp.alloc(&sel, std::max<uint32_t>(n_mine, 1)));
        if (n_mine) {
            HJ_CUDA(cudaMemcpyAsync(d_items, mine.data(), (size_t)n_mine * 4, cudaMemcpyHostToDevice, st));
            k_pick_list<<<(n_mine + 255) / 256, 256, 0, st>>>(blocks, d_items, n_mine, sel);
            HJ_LAUNCHED();
        }
        HJ_CUDA(cudaStreamSynchronize(st));   // the host copy of the item list is read by the copy above
        tmp.release(blocks);
        tmp.release(d_items);
        blocks = sel;
        nblocks = n_mine;
    }

    // the join's counters and flags: one allocation, reset per batch by one kernel and
    // read back with one copy
    JoinCtl* ctl = nullptr;
    HJ_TRY(tmp.alloc(&ctl, 1));
    HJ_CUDA(cudaMemsetAsync(ctl, 0, sizeof(JoinCtl), st));
    unsigned int* head = &ctl->head;
    uint32_t* overflow = &ctl->overflow;
    PairSink no_band{nullptr, nullptr, nullptr, 0, overflow};

    EventPairs kev;   // refine kernel launches of the join proper
    // head_reset: zero the work-item queue head first (batches reset it with the rest)
    auto run_refine = [&](const HjBlock* blk, uint32_t nb, const PairSink& sink, const PairSink& band,
                          uint32_t count_only, unsigned long long* bc, bool head_reset = true,
                          uint32_t* qcount = nullptr) -> hj_status {
        if (head_reset) HJ_CUDA(cudaMemsetAsync(head, 0, sizeof(unsigned int), st));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (!count_only) {
            kev.ev.emplace_back(nullptr, nullptr);
            HJ_TRY(event_acquire(&kev.ev.back().first));
            HJ_TRY(event_acquire(&kev.ev.back().second));
            e0 = kev.ev.back().first;
            e1 = kev.ev.back().second;
            HJ_CUDA(cudaEventRecord(e0, st));
        }
        HJ_TRY(tc ? launch_refine_tc(ix, blk, nb, head, sink, band, count_only, bc,
                                     count_only ? nullptr : &ctl->tc_acc, &ctl->timeout, st)
                  : launch_refine_plain(ix, blk, nb, head, sink, count_only, bc, qcount, st));
        if (!count_only) HJ_CUDA(cudaEventRecord(e1, st));
        return HJ_OK;
    };
    auto check_timeout = [&]() -> hj_status {
        uint32_t to = 0;
        HJ_CUDA(cudaMemcpyAsync(&to, &ctl->timeout, 4, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        if (to) {
            set_error("hj_join: a bounded device-side wait expired in the tensor-core pipeline");
            return HJ_ERR_TIMEOUT;
        }
        return HJ_OK;
    };

    // ---- estimator (GPUBatchEst_v2, GPU.cu:403-779)
    auto t_est = std::chrono::steady_clock::now();
    S.ms_setup = ms_since(t_start);
    uint32_t stride = std::max<uint32_t>(1, (uint32_t)std::lround(1.0 / opts.sample_rate));
    uint32_t nsamp = nblocks ? (nblocks + stride - 1) / stride : 0;
    {
        // a sample of a few persistent-kernel rounds ends with a partly filled round, which
        // costs as much as a full one: take whole rounds (a multiple of the SM count), at
        // most the requested rate
        const uint32_t sms = (uint32_t)num_sms();
        if (nsamp > sms && nsamp < 8 * sms) {
            const uint32_t want = (nsamp / sms) * sms;
            stride = (nblocks + want - 1) / want;
            nsamp = (nblocks + stride - 1) / stride;
        }
    }
    double total_est = 0, cand_total = 0;
    double* pest = nullptr;   // exclusive prefix of the per-item estimates (nblocks + 1)
    double* dsum = nullptr;
    if (nsamp) {
        HjBlock* sblocks = nullptr;
        unsigned long long* scnt = nullptr;
        HJ_TRY(tmp.alloc(&sblocks, nsamp));
        HJ_TRY(tmp.alloc(&scnt, nsamp));
        HJ_CUDA(cudaMemsetAsync(scnt, 0, nsamp * sizeof(unsigned long long), st));
        k_pick_samples<<<(nsamp + 255) / 256, 256, 0, st>>>(blocks, nblocks, stride, nsamp, sblocks);
        HJ_LAUNCHED();
        PairSink none{nullptr, nullptr, nullptr, 0, overflow};
        int tuned = 0;
        const std::string key = tune_key(refine, ix->d, ix->dtype);
        if (tc && !tune_lookup(key, &tuned) && tuning_enabled()) {
            // the vote form follows the hit density: measure it on the sample first, so the
            // shapes are timed in the form the refine will use
            HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
            HJ_TRY(check_timeout());
            {
                std::vector<unsigned long long> h0(nsamp);
                std::vector<HjBlock> hs0(nsamp);
                HJ_CUDA(cudaMemcpyAsync(h0.data(), scnt, nsamp * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                        st));
                HJ_CUDA(cudaMemcpyAsync(hs0.data(), sblocks, nsamp * sizeof(HjBlock), cudaMemcpyDeviceToHost, st));
                HJ_CUDA(cudaStreamSynchronize(st));
                double sp = 0, sc = 0;
                for (uint32_t q = 0; q < nsamp; ++q) {
                    sp += (double)h0[q];
                    sc += (double)hs0[q].nb * (hs0[q].q1 - hs0[q].q0);
                }
                tc_set_defer(ix, defer_for(sp, sc));
            }
            // time each epilogue shape on the sample; the last run's counts are the estimate.
            // Shapes: warp groups | 8 * (one warp set per accumulator)
            const int cands[4] = {2, 4, 10, 12};
            float best = 1e30f;
            int best_epi = tc_get_epi(ix);
            EventPairs tev;
            tev.ev.emplace_back(nullptr, nullptr);
            HJ_TRY(event_acquire(&tev.ev[0].first));
            HJ_TRY(event_acquire(&tev.ev[0].second));
            for (int c : cands) {
                tc_set_epi(ix, c);
                HJ_CUDA(cudaMemsetAsync(scnt, 0, nsamp * sizeof(unsigned long long), st));
                HJ_CUDA(cudaEventRecord(tev.ev[0].first, st));
                HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
                HJ_CUDA(cudaEventRecord(tev.ev[0].second, st));
                HJ_TRY(check_timeout());
                float ms = 0;
                HJ_CUDA(cudaEventElapsedTime(&ms, tev.ev[0].first, tev.ev[0].second));
                if (ms < best) { best = ms; best_epi = c; }
            }
            tc_set_epi(ix, best_epi);
            tune_store(key, best_epi);
        } else if (!tc && nsamp >= 16 && !tune_lookup(key, &tuned) && tuning_enabled()) {
            // the exact refine's two tile shapes, timed on the sample (each run twice, the
            // faster run kept: the first run of a shape also pays its one-time setup); the
            // last run's counts are the estimate, and they are the same for either shape
            float best = 1e30f;
            int best_shape = 0;
            EventPairs tev;
            tev.ev.emplace_back(nullptr, nullptr);
            HJ_TRY(event_acquire(&tev.ev[0].first));
            HJ_TRY(event_acquire(&tev.ev[0].second));
            for (int shape : {1, 0}) {
                ix->plain_shape = shape;
                for (int rep = 0; rep < 2; ++rep) {
                    HJ_CUDA(cudaMemsetAsync(scnt, 0, nsamp * sizeof(unsigned long long), st));
                    HJ_CUDA(cudaEventRecord(tev.ev[0].first, st));
                    HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
                    HJ_CUDA(cudaEventRecord(tev.ev[0].second, st));
                    HJ_CUDA(cudaEventSynchronize(tev.ev[0].second));
                    float ms = 0;
                    HJ_CUDA(cudaEventElapsedTime(&ms, tev.ev[0].first, tev.ev[0].second));
                    if (ms < best) { best = ms; best_shape = shape; }
                }
            }
            ix->plain_shape = best_shape;   // the exact counts of the last run do not depend on the shape
            tune_store(key, best_shape);
        } else {
            if (tc && tuned) tc_set_epi(ix, tuned);
            if (!tc) ix->plain_shape = tuned;
            HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
            HJ_TRY(check_timeout());
        }
        // per-item estimates and their exclusive prefix on the device; the host reads the
        // totals only (the item list of a sparse dataset runs to millions of entries)
        HJ_TRY(tmp.alloc(&pest, (size_t)nblocks + 1));
        HJ_TRY(tmp.alloc(&dsum, 1));
        HJ_CUDA(cudaMemsetAsync(dsum, 0, sizeof(double), st));
        k_item_estimates<<<(nblocks + 256) / 256, 256, 0, st>>>(blocks, nblocks, stride, nsamp, sblocks, scnt, pest,
                                                                 dsum);
        HJ_LAUNCHED();
        HJ_TRY(scan_f64_inplace(pest, (uint64_t)nblocks + 1, st));
        double hsum[2] = {0, 0};
        HJ_CUDA(cudaMemcpyAsync(&hsum[0], pest + nblocks, sizeof(double), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaMemcpyAsync(&hsum[1], dsum, sizeof(double), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        total_est = hsum[0];
        cand_total = hsum[1];
    }
    S.estimated_pairs = (uint64_t)total_est;
    S.ms_estimate = ms_since(t_est);
    if (tc) tc_set_defer(ix, defer_for(total_est, cand_total));

    // ---- result buffer capacity
    // slack for partly filled warp chunks: every warp that can emit during a batch holds
    // at most one (sized from the launch grids, so small joins get small buffers)
    const uint64_t chunk_slack = (tc ? tc_emit_warps(nblocks) : plain_emit_warps(nblocks)) * kSinkChunk;
    // keys, vals, their grouped copies (+ band pair ids; + a second set of grouped copies)
    const bool overlap = opts.stream_overlap && handler.can_overlap();
    const uint32_t base_words = tc ? 6u : 4u;
    const uint32_t slot_words = base_words + (overlap ? 2u : 0u);
    const double bytes_per_slot = 4.0 * slot_words;
    const uint64_t want = (uint64_t)(total_est * 2.0) + chunk_slack + 4096;
    uint64_t cap = opts.result_capacity ? opts.result_capacity + chunk_slack : want;
    if (cap < chunk_slack * 2) cap = chunk_slack * 2;
    const double result_bytes = kept_bytes_per_pair * total_est * 1.1;   // what the handler keeps
    S.bytes_wanted = (uint64_t)((double)cap * bytes_per_slot + result_bytes) + fixed_kept_bytes;
    // the caller's cap (a serving loop's reservation): smaller buffers mean more batches; a
    // join that cannot fit even two warp chunks per emitting warp beside its results is refused
    const uint64_t cap_bytes = opts.device_bytes_cap;
    if (cap_bytes) {
        const double room = (double)cap_bytes - (double)fixed_kept_bytes - result_bytes;
        const uint64_t fit = room > 0 ? (uint64_t)(room / bytes_per_slot) : 0;
        cap = std::min(cap, fit);
        if (cap < chunk_slack * 2) {
            set_error("hj_join: the join needs about %llu device bytes, more than its cap of %llu",
                      (unsigned long long)S.bytes_wanted, (unsigned long long)cap_bytes);
            if (stats) *stats = S;
            return HJ_ERR_OOM;
        }
    }
    // the device-wide free-memory query (a driver call) only when the buffers are large
    auto max_cap_from_free = [&](uint64_t* out) -> hj_status {
        size_t free_b = 0, total_b = 0;
        HJ_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const double usable = std::max(0.0, (double)free_b - result_bytes);
        *out = std::min<uint64_t>((uint64_t)(opts.mem_fraction * usable / bytes_per_slot), 0xF0000000ull);
        return HJ_OK;
    };
    const bool large = (double)cap * bytes_per_slot + result_bytes > 1024.0 * 1024 * 1024;
    if (large) {
        uint64_t max_cap = 0;
        HJ_TRY(max_cap_from_free(&max_cap));
        cap = std::min(cap, max_cap);
    }
    cap = std::min<uint64_t>(cap, 0xF0000000ull);   // radix sort and 32-bit counts per batch
    if (cap <= chunk_slack) {
        set_error("hj_join: not enough device memory for a result buffer");
        return HJ_ERR_OOM;
    }

    // ---- batches: cut the workload order at half the buffer by estimate
    std::vector<Batch> batches;
    if (nblocks) {
        const double budget = 0.5 * (double)(cap - chunk_slack);
        std::vector<uint32_t> cuts;
        if (nblocks > 1 && total_est >= budget) {
            uint32_t* dcuts = nullptr;
            unsigned int* dn = nullptr;
            HJ_TRY(tmp.alloc(&dcuts, nblocks));
            HJ_TRY(tmp.alloc(&dn, 1));
            HJ_CUDA(cudaMemsetAsync(dn, 0, sizeof(unsigned int), st));
            k_batch_cuts<<<(nblocks + 254) / 256, 256, 0, st>>>(pest, nblocks, budget, dcuts, dn);
            HJ_LAUNCHED();
            unsigned int ncut = 0;
            HJ_CUDA(cudaMemcpyAsync(&ncut, dn, sizeof(ncut), cudaMemcpyDeviceToHost, st));
            HJ_CUDA(cudaStreamSynchronize(st));
            cuts.resize(ncut);
            if (ncut) {
                HJ_CUDA(cudaMemcpyAsync(cuts.data(), dcuts, (size_t)ncut * 4, cudaMemcpyDeviceToHost, st));
                HJ_CUDA(cudaStreamSynchronize(st));
            }
            std::sort(cuts.begin(), cuts.end());
        }
        uint32_t b0 = 0;
        for (uint32_t c : cuts) {
            batches.push_back({b0, c});
            b0 = c;
        }
        batches.push_back({b0, nblocks});
    }
    std::reverse(batches.begin(), batches.end());   // used as a stack

    // one allocation carved into keys, vals, their radix copies and the band pair ids;
    // when the free-memory query was skipped and the allocation fails, query and retry smaller
    uint32_t* slab = nullptr;
    hj_status as = tmp.alloc(&slab, cap * slot_words);
    if (as == HJ_ERR_OOM && !large && !opts.result_capacity) {
        uint64_t max_cap = 0;
        HJ_TRY(max_cap_from_free(&max_cap));
        if (max_cap < cap && max_cap > chunk_slack) {
            cap = max_cap;
            as = tmp.alloc(&slab, cap * slot_words);
        }
    }
    HJ_TRY(as);
    uint32_t *keys = slab, *vals = slab + cap, *keys_tmp = slab + 2 * cap, *vals_tmp = slab + 3 * cap;
    uint32_t* band_q = tc ? slab + 4 * cap : nullptr;
    uint32_t* band_c = tc ? slab + 5 * cap : nullptr;
    // the grouped copies, one set per batch parity with stream_overlap
    uint32_t* grp_keys[2] = {keys_tmp, overlap ? slab + (size_t)base_words * cap : keys_tmp};
    uint32_t* grp_vals[2] = {vals_tmp, overlap ? slab + (size_t)(base_words + 1) * cap : vals_tmp};
    cudaEvent_t release[2] = {nullptr, nullptr};   // a sink's events: the set is still being read
    uint32_t* qoff = nullptr;   // per-query counters, then first slots, of the grouping
    HJ_TRY(tmp.alloc(&qoff, (size_t)ix->n + 1));
    // the exact refine counts each query's pairs itself when every item takes its block path
    // (no warp path below k = 4): the grouping then skips its counting pass
    const bool fused_counts = !tc && plain_counts_queries(ix);

    auto t_ref = std::chrono::steady_clock::now();
    float ms_group = 0;
    uint64_t total = 0;
    double kept = (double)fixed_kept_bytes + (double)cap * bytes_per_slot;   // against the cap
    uint32_t n_out = 0;
    while (!batches.empty()) {
        Batch b = batches.back();
        batches.pop_back();
        if (opts.max_batches && n_out >= opts.max_batches) {
            set_error("hj_join: batch limit %u reached", opts.max_batches);
            return HJ_ERR_OVERFLOW;
        }
        k_batch_reset<<<1, 32, 0, st>>>(ctl);
        HJ_LAUNCHED();
        PairSink sink{keys, vals, &ctl->cursor, cap, overflow};
        PairSink band = tc ? PairSink{band_q, band_c, &ctl->band_cursor, cap, overflow} : no_band;
        if (fused_counts) HJ_CUDA(cudaMemsetAsync(qoff, 0, ((size_t)ix->n + 1) * 4, st));
        HJ_TRY(run_refine(blocks + b.b0, b.b1 - b.b0, sink, band, 0, nullptr, false, fused_counts ? qoff : nullptr));
        if (tc) HJ_TRY(launch_band_recheck(ix, band_q, band_c, &ctl->band_cursor, cap, sink, b.b1 - b.b0, st));
        JoinCtl hc;
        HJ_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof(JoinCtl), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        if (hc.timeout) {
            set_error("hj_join: a bounded device-side wait expired in the tensor-core pipeline");
            return HJ_ERR_TIMEOUT;
        }
        const unsigned long long used = hc.cursor;
        if (hc.overflow) {
            if (b.b1 - b.b0 <= 1) {
                set_error("hj_join: one work item produces more pairs than the result buffer holds (%llu)",
                          (unsigned long long)cap);
                return HJ_ERR_OVERFLOW;
            }
            uint32_t mid = b.b0 + (b.b1 - b.b0) / 2;
            batches.push_back({mid, b.b1});
            batches.push_back({b.b0, mid});
            S.n_retries++;
            continue;
        }
        S.tc_accepts += hc.tc_acc;
        S.band_pairs += hc.tc_band;
        auto t_g = std::chrono::steady_clock::now();
        const uint64_t slots = std::min<uint64_t>(used, cap);
        uint32_t valid = 0;
        if (slots) {
            // group by query id: count (unless the refine counted), scan (qoff[n] = the batch's
            // pairs), scatter into the copies
            const unsigned g = (unsigned)std::min<uint64_t>((slots + kGrpTile - 1) / kGrpTile, (uint64_t)num_sms() * 8);
            if (!fused_counts) {
                HJ_CUDA(cudaMemsetAsync(qoff, 0, ((size_t)ix->n + 1) * 4, st));
                k_group_count<<<g, 256, 0, st>>>(keys, slots, qoff);
                HJ_LAUNCHED();
            }
            HJ_TRY(scan_u32_inplace(qoff, (uint64_t)ix->n + 1, st));
            HJ_CUDA(cudaMemcpyAsync(&valid, qoff + ix->n, 4, cudaMemcpyDeviceToHost, st));
            const int set = overlap ? (int)(n_out & 1u) : 0;
            if (release[set]) {   // the sink's reads of this set, two batches ago
                HJ_CUDA(cudaStreamWaitEvent(st, release[set], 0));
                release[set] = nullptr;
            }
            k_group_scatter<<<g, 256, 0, st>>>(keys, vals, slots, qoff, grp_keys[set], grp_vals[set]);
            HJ_LAUNCHED();
            HJ_CUDA(cudaStreamSynchronize(st));
        }
        if (cap_bytes && kept + kept_bytes_per_pair * (double)valid > (double)cap_bytes) {
            // the estimate was low: refuse before the results pass the cap, asking for the
            // results so far extrapolated over the remaining work items (heaviest first, so
            // this errs high)
            const double slab_b = (double)cap * bytes_per_slot;
            const double so_far = kept - (double)fixed_kept_bytes - slab_b + kept_bytes_per_pair * (double)valid;
            const double frac = (double)std::max<uint32_t>(1, b.b1) / nblocks;
            S.bytes_wanted = std::max<uint64_t>(
                S.bytes_wanted, (uint64_t)((double)fixed_kept_bytes + slab_b + 1.1 * so_far / frac));
            set_error("hj_join: the results outgrow the cap of %llu device bytes",
                      (unsigned long long)cap_bytes);
            if (stats) *stats = S;
            return HJ_ERR_OOM;
        }
        kept += kept_bytes_per_pair * (double)valid;
        {
            const int set = overlap ? (int)(n_out & 1u) : 0;
            if (release[set]) {   // an empty batch reuses the set without a scatter
                HJ_CUDA(cudaStreamWaitEvent(st, release[set], 0));
                release[set] = nullptr;
            }
            HJ_TRY(handler.on_batch(n_out, grp_keys[set], grp_vals[set], valid, valid ? qoff : nullptr, st));
            release[set] = handler.take_release();
        }
        ++n_out;
        total += valid;
        ms_group += ms_since(t_g);
    }
    for (cudaEvent_t e : release)
        if (e) HJ_CUDA(cudaStreamWaitEvent(st, e, 0));   // the sink's last reads end before the join does
    HJ_CUDA(cudaStreamSynchronize(st));
    S.ms_refine = ms_since(t_ref) - ms_group;
    S.ms_group = ms_group;
    for (auto& ev : kev.ev) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess) S.ms_refine_kernel += ms;
        S.refine_launches++;
    }
    cudaGetLastError();
    S.total_pairs = total;
    S.n_batches = n_out;
    S.ms_total = ms_since(t_start);
    S.kernel_launches = (uint32_t)(thread_launch_count() - launches0);
    if (stats) *stats = S;
    return HJ_OK;
}

// hj_join: every batch's neighbour ids stay on the device (a copy per batch) and
// the device neighbour table points into them.
struct RetainHandler : BatchHandler {
    hj_result* res;
    bool keep_keys;
    RetainHandler(hj_result* r, bool kk) : res(r), keep_keys(kk) {}
    hj_status on_batch(uint32_t bi, const uint32_t* keys, const uint32_t* vals, uint64_t count,
                       const uint32_t* run_end, cudaStream_t st) override {
        uint32_t* bv = nullptr;
        HJ_TRY(dalloc(&bv, count, st));
        res->vals.push_back(bv);
        res->counts.push_back(count);
        if (count) HJ_CUDA(cudaMemcpyAsync(bv, vals, count * 4, cudaMemcpyDeviceToDevice, st));
        if (keep_keys) {
            uint32_t* bk = nullptr;
            HJ_TRY(dalloc(&bk, count, st));
            res->keys.push_back(bk);
            if (count) HJ_CUDA(cudaMemcpyAsync(bk, keys, count * 4, cudaMemcpyDeviceToDevice, st));
        }
        if (count) {
            k_table_runs<<<(res->n + 255) / 256, 256, 0, st>>>(run_end, res->n, bi, res->table);
            HJ_LAUNCHED();
        }
        res->total += count;
        return HJ_OK;
    }
};

// hj_join_stream: per-query digests accumulated on the device, then the caller's
// sink; nothing is kept after the sink returns.
struct StreamHandler : BatchHandler {
    hj_batch_sink sink;
    void* user;
    uint32_t* cnt;
    unsigned long long* sum;
    unsigned long long* xr;
    StreamHandler(hj_batch_sink s, void* u, uint32_t* c, uint64_t* sm, uint64_t* x)
        : sink(s), user(u), cnt(c), sum(reinterpret_cast<unsigned long long*>(sm)),
          xr(reinterpret_cast<unsigned long long*>(x)) {}
    hj_status on_batch(uint32_t bi, const uint32_t* keys, const uint32_t* vals, uint64_t count,
                       const uint32_t* /*run_end*/, cudaStream_t st) override {
        if (count && cnt) {
            const uint64_t per_block = 8ull * kDigestSpan;   // 8 warps, each a walk of 512 pairs
            const unsigned g = (unsigned)std::min<uint64_t>((count + per_block - 1) / per_block, (uint64_t)num_sms() * 16);
            k_digest_accumulate<<<g, 256, 0, st>>>(keys, vals, count, cnt, sum, xr);
            HJ_LAUNCHED();
        }
        if (!sink) return HJ_OK;
        hj_batch_view v{bi, 0u, count, keys, vals, nullptr};
        hj_status s = sink(&v, user, st);
        last_release = static_cast<cudaEvent_t>(v.release_event);
        if (s != HJ_OK) {
            set_error("hj_join_stream: the batch sink returned %d", s);
            return s;
        }
        return HJ_OK;
    }
    bool can_overlap() const override { return sink != nullptr; }
    cudaEvent_t take_release() override {
        cudaEvent_t e = last_release;
        last_release = nullptr;
        return e;
    }
    cudaEvent_t last_release = nullptr;
};

}  // namespace
}  // namespace hj

using namespace hj;

extern "C" {

hj_status hj_shard_plan(uint32_t n_items, uint32_t shard_count, uint32_t shard_index, uint32_t* first,
                        uint32_t* stride, uint32_t* n_mine) {
    if (shard_count == 0 || shard_index >= shard_count || !first || !stride || !n_mine) {
        set_error("hj_shard_plan: shard_index %u out of range for %u shards", shard_index, shard_count);
        return HJ_ERR_INVALID;
    }
    // round robin over the heaviest-first order
    *first = shard_index;
    *stride = shard_count;
    *n_mine = n_items > shard_index ? (n_items - shard_index + shard_count - 1) / shard_count : 0;
    return HJ_OK;
}

hj_status hj_shard_plan_lpt(const uint64_t* costs, uint32_t n_items, uint32_t shard_count, uint32_t shard_index,
                            uint32_t* items, uint32_t* n_mine) {
    if (shard_count == 0 || shard_index >= shard_count || !n_mine || (n_items && (!costs || !items))) {
        set_error("hj_shard_plan_lpt: invalid arguments (%u items, shard %u of %u)", n_items, shard_index,
                  shard_count);
        return HJ_ERR_INVALID;
    }
    // longest processing time first: items by cost, descending (ties by index), each to
    // the least-loaded shard (ties to the lowest shard index); every rank computes the
    // same assignment from the same costs
    std::vector<uint32_t> order(n_items);
    for (uint32_t i = 0; i < n_items; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return costs[a] > costs[b]; });
    using Load = std::pair<uint64_t, uint32_t>;   // (load, shard)
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (uint32_t s = 0; s < shard_count; ++s) heap.push({0, s});
    std::vector<uint8_t> mine(n_items, 0);
    for (uint32_t i : order) {
        Load l = heap.top();
        heap.pop();
        if (l.second == shard_index) mine[i] = 1;
        l.first += costs[i];
        heap.push(l);
    }
    uint32_t m = 0;
    for (uint32_t i = 0; i < n_items; ++i)
        if (mine[i]) items[m++] = i;   // ascending: the heaviest-first order within the shard
    *n_mine = m;
    return HJ_OK;
}

void hj_join_opts_default(hj_join_opts* o) {
    if (!o) return;
    *o = hj_join_opts{};
    o->refine = HJ_REFINE_AUTO;
    o->sample_rate = 0.02;
    o->mem_fraction = 0.6;
    o->use_graphs = 0;
    o->keep_keys = 0;
}

hj_status hj_result_destroy(hj_result* r) {
    if (!r) return HJ_OK;
    for (auto* p : r->vals) cudaFreeAsync(p, r->stream);
    for (auto* p : r->keys) cudaFreeAsync(p, r->stream);
    if (r->d_batch_vals) cudaFreeAsync(r->d_batch_vals, r->stream);
    if (r->table) cudaFreeAsync(r->table, r->stream);
    delete r;
    return HJ_OK;
}

hj_status hj_join(hj_index* ix, const hj_join_opts* opts, void* stream, hj_result** out, hj_join_stats* stats) {
    if (!ix || !out) { set_error("hj_join: null argument"); return HJ_ERR_INVALID; }
    *out = nullptr;
    cudaStream_t st = as_stream(stream);
    hj_result* res = new hj_result();
    res->n = ix->n;
    res->stream = st;
    hj_status s = dalloc(&res->table, ix->n, st);
    if (s == HJ_OK) s = cuda_status(cudaMemsetAsync(res->table, 0, (size_t)ix->n * sizeof(hj_nt_entry), st),
                                    "clear the neighbour table");
    const bool keep_keys = opts && opts->keep_keys;
    RetainHandler h(res, keep_keys);
    hj_join_stats S{};
    if (s == HJ_OK) s = join_impl(ix, opts, st, h, keep_keys ? 8.0 : 4.0, (uint64_t)ix->n * sizeof(hj_nt_entry), &S);
    if (s == HJ_OK && !res->vals.empty()) {
        s = dalloc(&res->d_batch_vals, res->vals.size(), st);
        if (s == HJ_OK)
            s = cuda_status(cudaMemcpyAsync(res->d_batch_vals, res->vals.data(), res->vals.size() * sizeof(uint32_t*),
                                            cudaMemcpyHostToDevice, st), "batch pointer table");
    }
    if (s == HJ_OK) s = cuda_status(cudaStreamSynchronize(st), "hj_join");
    if (stats) *stats = S;   // on an error: what was known (bytes_wanted when the cap refused)
    if (s != HJ_OK) {
        hj_result_destroy(res);
        return s;
    }
    *out = res;
    return HJ_OK;
}

hj_status hj_join_stream(hj_index* ix, const hj_join_opts* opts, hj_batch_sink sink, void* user, uint32_t* d_count,
                         uint64_t* d_sum, uint64_t* d_xor, void* stream, hj_join_stats* stats) {
    if (!ix) { set_error("hj_join_stream: null index"); return HJ_ERR_INVALID; }
    if ((d_count != nullptr) != (d_sum != nullptr) || (d_count != nullptr) != (d_xor != nullptr)) {
        set_error("hj_join_stream: pass all three digest arrays or none");
        return HJ_ERR_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    if (d_count) {
        HJ_CUDA(cudaMemsetAsync(d_count, 0, (size_t)ix->n * 4, st));
        HJ_CUDA(cudaMemsetAsync(d_sum, 0, (size_t)ix->n * 8, st));
        HJ_CUDA(cudaMemsetAsync(d_xor, 0, (size_t)ix->n * 8, st));
    }
    StreamHandler h(sink, user, d_count, d_sum, d_xor);
    HJ_TRY(join_impl(ix, opts, st, h, 0.0, 0, stats));
    HJ_CUDA(cudaStreamSynchronize(st));
    return HJ_OK;
}

hj_status hj_result_num_batches(const hj_result* r, uint32_t* nb, uint64_t* total) {
    if (!r) { set_error("hj_result_num_batches: null result"); return HJ_ERR_INVALID; }
    if (nb) *nb = (uint32_t)r->vals.size();
    if (total) *total = r->total;
    return HJ_OK;
}

hj_status hj_result_batch(const hj_result* r, uint32_t b, const uint32_t** v, const uint32_t** k, uint64_t* count) {
    if (!r || b >= r->vals.size()) { set_error("hj_result_batch: bad batch index"); return HJ_ERR_INVALID; }
    if (v) *v = r->vals[b];
    if (k) *k = r->keys.empty() ? nullptr : r->keys[b];
    if (count) *count = r->counts[b];
    return HJ_OK;
}

hj_status hj_result_table(const hj_result* r, const hj_nt_entry** t) {
    if (!r || !t) { set_error("hj_result_table: null argument"); return HJ_ERR_INVALID; }
    *t = r->table;
    return HJ_OK;
}

hj_status hj_result_to_csr(const hj_result* r, uint64_t* d_off, uint32_t* d_vals, int sort_lists, void* stream) {
    if (!r || !d_off) { set_error("hj_result_to_csr: null argument"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    uint32_t n = r->n;
    uint32_t* cnt = nullptr;
    HJ_TRY(dalloc(&cnt, (size_t)n + 1, st));
    k_table_counts<<<(n + 255) / 256, 256, 0, st>>>(r->table, n, cnt);
    HJ_LAUNCHED();
    HJ_CUDA(cudaMemsetAsync(cnt + n, 0, 4, st));
    HJ_TRY(scan_u32_to_u64(cnt, d_off, (uint64_t)n + 1, st));
    dfree(cnt, st);
    if (!d_vals || r->total == 0) return HJ_OK;
    unsigned g = (unsigned)(((uint64_t)n * 32 + 255) / 256);
    k_csr_copy<<<g, 256, 0, st>>>(r->table, r->d_batch_vals, n, d_off, d_vals);
    HJ_LAUNCHED();
    if (sort_lists) {
        uint64_t P = r->total;
        uint64_t *k64 = nullptr, *k64t = nullptr;
        uint32_t *v = nullptr, *vt = nullptr;
        HJ_TRY(dalloc(&k64, P, st));
        HJ_TRY(dalloc(&k64t, P, st));
        HJ_TRY(dalloc(&v, P, st));
        HJ_TRY(dalloc(&vt, P, st));
        k_csr_keys<<<g, 256, 0, st>>>(r->table, d_vals, n, d_off, k64);
        HJ_LAUNCHED();
        HJ_CUDA(cudaMemsetAsync(v, 0, P * 4, st));
        HJ_TRY(radix_sort_u64_u32(k64, v, k64t, vt, P, 32 + bits_for(n), st));
        k_unpack_vals<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(k64, P, d_vals);
        HJ_LAUNCHED();
        dfree(k64, st); dfree(k64t, st); dfree(v, st); dfree(vt, st);
    }
    return HJ_OK;
}

hj_status hj_result_digest(const hj_result* r, uint32_t* d_count, uint64_t* d_sum, uint64_t* d_xor, void* stream) {
    if (!r) { set_error("hj_result_digest: null result"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    unsigned g = (unsigned)(((uint64_t)r->n * 32 + 255) / 256);
    k_digest<<<g, 256, 0, st>>>(r->table, r->d_batch_vals, r->n, d_count, d_sum, d_xor);
    HJ_LAUNCHED();
    return HJ_OK;
}

hj_status hj_self_join_host(const void* h_db, uint32_t n, uint32_t d, uint32_t k, int dtype, double eps,
                            const hj_join_opts* opts, void* stream, hj_result** out, hj_join_stats* stats) {
    if (!h_db || n == 0 || d == 0) { set_error("hj_self_join_host: invalid arguments"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    size_t bytes = (size_t)n * d * (dtype == HJ_F64 ? 8 : 4);
    void* d_db = nullptr;
    HJ_CUDA(cudaMallocAsync(&d_db, bytes, st));
    HJ_CUDA(cudaMemcpyAsync(d_db, h_db, bytes, cudaMemcpyHostToDevice, st));
    hj_index* ix = nullptr;
    hj_status s = hj_index_create(d_db, n, d, k, dtype, eps, nullptr, nullptr, stream, &ix);
    cudaFreeAsync(d_db, st);
    if (s != HJ_OK) return s;
    hj_result* r = nullptr;
    s = hj_join(ix, opts, stream, &r, stats);
    hj_index_destroy(ix);
    if (s != HJ_OK) return s;
    if (out) *out = r; else hj_result_destroy(r);
    return HJ_OK;
}

}  // extern "C"
