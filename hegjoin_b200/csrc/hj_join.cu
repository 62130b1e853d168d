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
#include <sstream>

#include "hj_internal.h"

namespace hj {
uint32_t plain_query_block(int dtype);
hj_status launch_refine_plain(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                              const PairSink& sink, uint32_t count_only, unsigned long long* block_counts,
                              cudaStream_t st);
hj_status tc_prepare(hj_index* ix, int kind, cudaStream_t st);
uint32_t tc_query_block();
hj_status launch_refine_tc(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                           const PairSink& sink, const PairSink& band, uint32_t count_only,
                           unsigned long long* block_counts, unsigned long long* stats, uint32_t* err,
                           cudaStream_t st);
hj_status launch_band_recheck(const hj_index* ix, const uint32_t* bq, const uint32_t* bc,
                              const unsigned long long* band_used, unsigned long long band_cap,
                              const PairSink& sink, cudaStream_t st);
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

__global__ void k_pick_strided(const HjBlock* __restrict__ blocks, uint32_t first, uint32_t stride, uint32_t m,
                               HjBlock* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = blocks[first + i * stride];
}

// Number of non-sentinel keys in a sorted key array (sentinels sort last).
__global__ void k_count_valid(const uint32_t* __restrict__ keys, unsigned long long n, unsigned long long* out) {
    unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool v = keys[i] != kSentinelKey;
    bool nxt = (i + 1 < n) && keys[i + 1] != kSentinelKey;
    if (v && !nxt) *out = i + 1;
}

__device__ __forceinline__ unsigned long long lower_bound_u32(const uint32_t* a, unsigned long long n, uint32_t v) {
    unsigned long long lo = 0, hi = n;
    while (lo < hi) {
        unsigned long long mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// constructNeighborTableKeyValueWithPtrs (GPU.cu:1731-1776) on the device: one
// entry per run of equal keys, written by the run's last element.
__global__ void k_table(const uint32_t* __restrict__ keys, unsigned long long n, uint32_t batch,
                        hj_nt_entry* __restrict__ table) {
    unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t key = keys[i];
    if (i + 1 == n || keys[i + 1] != key) {
        unsigned long long lo = lower_bound_u32(keys, i + 1, key);
        table[key] = hj_nt_entry{batch, (uint32_t)(i + 1 - lo), lo};
    }
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
}  // namespace hj

using namespace hj;

extern "C" {

hj_status hj_shard_plan(uint32_t n_items, uint32_t shard_count, uint32_t shard_index, uint32_t* first,
                        uint32_t* stride, uint32_t* n_mine) {
    if (shard_count == 0 || shard_index >= shard_count || !first || !stride || !n_mine) {
        set_error("hj_shard_plan: shard_index %u out of range for %u shards", shard_index, shard_count);
        return HJ_ERR_INVALID;
    }
    // round robin over the heaviest-first order: every rank gets a mix of heavy
    // and light items (an LPT-like balance without a host pass over item costs)
    *first = shard_index;
    *stride = shard_count;
    *n_mine = n_items > shard_index ? (n_items - shard_index + shard_count - 1) / shard_count : 0;
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

hj_status hj_join(hj_index* ix, const hj_join_opts* opts_in, void* stream, hj_result** out, hj_join_stats* stats) {
    auto t_start = std::chrono::steady_clock::now();
    if (!ix || !out) { set_error("hj_join: null argument"); return HJ_ERR_INVALID; }
    *out = nullptr;
    hj_join_opts opts;
    if (opts_in) opts = *opts_in; else hj_join_opts_default(&opts);
    if (opts.sample_rate <= 0 || opts.sample_rate > 1) opts.sample_rate = 0.02;
    if (opts.mem_fraction <= 0 || opts.mem_fraction > 0.95) opts.mem_fraction = 0.6;
    cudaStream_t st = as_stream(stream);
    uint64_t launches0 = thread_launch_count();
    hj_join_stats S{};
    HJ_TRY(hj_sort_by_workload(ix, stream, nullptr));

    // ---- refine kind
    int refine = opts.refine;
    const bool auto_kind = refine == HJ_REFINE_AUTO;
    if (auto_kind)
        refine = (ix->dtype == HJ_F32 && ix->d >= 16 && tc_supported(ix, HJ_REFINE_TC_F16)) ? HJ_REFINE_TC_F16
                                                                                            : HJ_REFINE_EXACT;
    bool tc = refine == HJ_REFINE_TC_F16 || refine == HJ_REFINE_TC_BF16;
    if (tc) {
        if (!tc_supported(ix, refine)) {
            set_error("hj_join: the tensor-core filter needs float data with 16 <= d <= %d", 252);
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
    uint32_t qb = opts.query_block ? opts.query_block : (tc ? tc_query_block() : plain_query_block(ix->dtype));
    if (tc) qb = tc_query_block();   // the tensor-core tile shape fixes the block size
    if (!tc && qb != plain_query_block(ix->dtype)) qb = plain_query_block(ix->dtype);

    HjBlock* blocks = nullptr;
    uint32_t nblocks = 0;
    HJ_TRY(build_blocks(ix, qb, &blocks, &nblocks, st));
    if (opts.shard_count > 1) {
        // this rank's share of the heaviest-first order
        uint32_t first = 0, stride = 1, mine = 0;
        HJ_TRY(hj_shard_plan(nblocks, opts.shard_count, opts.shard_index, &first, &stride, &mine));
        HjBlock* sel = nullptr;
        HJ_TRY(dalloc(&sel, std::max<uint32_t>(mine, 1), st));
        if (mine) {
            k_pick_strided<<<(mine + 255) / 256, 256, 0, st>>>(blocks, first, stride, mine, sel);
            HJ_LAUNCHED();
        }
        dfree(blocks, st);
        blocks = sel;
        nblocks = mine;
    }

    unsigned int* head = nullptr;
    // [0] pair cursor, [1] valid count, [2] tc accepts, [3] tc band pairs, [4] band cursor
    unsigned long long* counters = nullptr;
    uint32_t* flags = nullptr;                 // [0] overflow, [1] bounded-wait timeout
    HJ_TRY(dalloc(&head, 1, st));
    HJ_TRY(dalloc(&counters, 8, st));
    HJ_TRY(dalloc(&flags, 2, st));
    HJ_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), st));
    HJ_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(uint32_t), st));
    uint32_t* overflow = flags;
    PairSink no_band{nullptr, nullptr, nullptr, 0, overflow};

    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kev;   // refine kernel launches of the join proper
    auto run_refine = [&](const HjBlock* blk, uint32_t nb, const PairSink& sink, const PairSink& band,
                          uint32_t count_only, unsigned long long* bc) -> hj_status {
        HJ_CUDA(cudaMemsetAsync(head, 0, sizeof(unsigned int), st));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (!count_only) {
            HJ_CUDA(cudaEventCreate(&e0));
            HJ_CUDA(cudaEventCreate(&e1));
            HJ_CUDA(cudaEventRecord(e0, st));
        }
        hj_status r = tc ? launch_refine_tc(ix, blk, nb, head, sink, band, count_only, bc,
                                            count_only ? nullptr : counters + 2, flags + 1, st)
                         : launch_refine_plain(ix, blk, nb, head, sink, count_only, bc, st);
        if (!count_only) {
            HJ_CUDA(cudaEventRecord(e1, st));
            kev.emplace_back(e0, e1);
        }
        return r;
    };
    auto check_timeout = [&]() -> hj_status {
        uint32_t to = 0;
        HJ_CUDA(cudaMemcpyAsync(&to, flags + 1, 4, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        if (to) {
            set_error("hj_join: a bounded device-side wait expired in the tensor-core pipeline");
            return HJ_ERR_TIMEOUT;
        }
        return HJ_OK;
    };

    // ---- estimator (GPUBatchEst_v2, GPU.cu:403-779)
    auto t_est = std::chrono::steady_clock::now();
    std::vector<HjBlock> hblocks(nblocks);
    if (nblocks) HJ_CUDA(cudaMemcpyAsync(hblocks.data(), blocks, (size_t)nblocks * sizeof(HjBlock), cudaMemcpyDeviceToHost, st));
    uint32_t stride = std::max<uint32_t>(1, (uint32_t)std::lround(1.0 / opts.sample_rate));
    uint32_t nsamp = nblocks ? (nblocks + stride - 1) / stride : 0;
    std::vector<double> est(nblocks, 0.0);
    double total_est = 0;
    if (nsamp) {
        HjBlock* sblocks = nullptr;
        unsigned long long* scnt = nullptr;
        HJ_TRY(dalloc(&sblocks, nsamp, st));
        HJ_TRY(dalloc(&scnt, nsamp, st));
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
                HJ_CUDA(cudaMemcpyAsync(h0.data(), scnt, nsamp * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                        st));
                HJ_CUDA(cudaStreamSynchronize(st));   // also completes the copy of hblocks
                double sp = 0, sc = 0;
                for (uint32_t q = 0; q < nsamp; ++q) {
                    const HjBlock& b = hblocks[std::min(nblocks - 1, q * stride)];
                    sp += (double)h0[q];
                    sc += (double)b.nb * (b.q1 - b.q0);
                }
                tc_set_defer(ix, defer_for(sp, sc));
            }
            // time each epilogue shape on the sample; the last run's counts are the estimate.
            // Shapes: warp groups | 8 * (one warp set per accumulator)
            const int cands[4] = {2, 4, 10, 12};
            float best = 1e30f;
            int best_epi = tc_get_epi(ix);
            cudaEvent_t e0, e1;
            HJ_CUDA(cudaEventCreate(&e0));
            HJ_CUDA(cudaEventCreate(&e1));
            for (int c : cands) {
                tc_set_epi(ix, c);
                HJ_CUDA(cudaMemsetAsync(scnt, 0, nsamp * sizeof(unsigned long long), st));
                HJ_CUDA(cudaEventRecord(e0, st));
                HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
                HJ_CUDA(cudaEventRecord(e1, st));
                HJ_TRY(check_timeout());
                float ms = 0;
                HJ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) { best = ms; best_epi = c; }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            tc_set_epi(ix, best_epi);
            tune_store(key, best_epi);
        } else {
            if (tc && tuned) tc_set_epi(ix, tuned);
            HJ_TRY(run_refine(sblocks, nsamp, none, no_band, 1, scnt));
            HJ_TRY(check_timeout());
        }
        std::vector<unsigned long long> hs(nsamp);
        HJ_CUDA(cudaMemcpyAsync(hs.data(), scnt, nsamp * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        dfree(sblocks, st);
        dfree(scnt, st);
        std::vector<double> rate(nsamp);
        for (uint32_t s = 0; s < nsamp; ++s) {
            const HjBlock& b = hblocks[std::min(nblocks - 1, s * stride)];
            rate[s] = (double)hs[s] / std::max<uint32_t>(1, b.q1 - b.q0);
        }
        for (uint32_t i = 0; i < nblocks; ++i) {
            uint32_t s = i / stride;
            double r = (i % stride == 0) ? rate[s] : std::max(rate[s], rate[std::min(nsamp - 1, s + 1)]);
            est[i] = r * (hblocks[i].q1 - hblocks[i].q0);
            total_est += est[i];
        }
    } else {
        HJ_CUDA(cudaStreamSynchronize(st));
    }
    S.estimated_pairs = (uint64_t)total_est;
    S.ms_estimate = ms_since(t_est);
    if (tc) {
        double cand = 0;
        for (uint32_t i = 0; i < nblocks; ++i) cand += (double)hblocks[i].nb * (hblocks[i].q1 - hblocks[i].q0);
        tc_set_defer(ix, defer_for(total_est, cand));
    }

    // ---- result buffer capacity
    size_t free_b = 0, total_b = 0;
    HJ_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const uint64_t chunk_slack = (uint64_t)num_sms() * 64 * kSinkChunk;   // partially filled warp chunks
    const double bytes_per_slot = 16.0 + 4.0 + (opts.keep_keys ? 4.0 : 0.0) + (tc ? 8.0 : 0.0);
    // leave room for the result itself (4 bytes per estimated pair, kept on the device)
    const double result_bytes = 4.0 * total_est * (opts.keep_keys ? 2.0 : 1.0) * 1.1;
    const double usable = std::max(0.0, (double)free_b - result_bytes);
    uint64_t max_cap = (uint64_t)(opts.mem_fraction * usable / bytes_per_slot);
    max_cap = std::min<uint64_t>(max_cap, 0xF0000000ull);
    uint64_t want = (uint64_t)(total_est * 2.0) + chunk_slack + 4096;
    uint64_t cap = opts.result_capacity ? opts.result_capacity + chunk_slack : std::min(want, max_cap);
    if (cap < chunk_slack * 2) cap = std::min<uint64_t>(chunk_slack * 2, max_cap);
    if (cap <= chunk_slack) {
        set_error("hj_join: not enough device memory for a result buffer");
        return HJ_ERR_OOM;
    }

    // ---- batches: cut the workload order at half the buffer by estimate
    std::vector<Batch> batches;
    {
        double budget = 0.5 * (double)(cap - chunk_slack);
        uint32_t b0 = 0;
        double run = 0;
        for (uint32_t i = 0; i < nblocks; ++i) {
            if (run > 0 && run + est[i] > budget) {
                batches.push_back({b0, i});
                b0 = i;
                run = 0;
            }
            run += est[i];
        }
        if (b0 < nblocks) batches.push_back({b0, nblocks});
    }
    std::reverse(batches.begin(), batches.end());   // used as a stack

    uint32_t *keys = nullptr, *vals = nullptr, *keys_tmp = nullptr, *vals_tmp = nullptr;
    uint32_t *band_q = nullptr, *band_c = nullptr;
    HJ_TRY(dalloc(&keys, cap, st));
    HJ_TRY(dalloc(&vals, cap, st));
    HJ_TRY(dalloc(&keys_tmp, cap, st));
    HJ_TRY(dalloc(&vals_tmp, cap, st));
    if (tc) {
        HJ_TRY(dalloc(&band_q, cap, st));
        HJ_TRY(dalloc(&band_c, cap, st));
    }

    hj_result* res = new hj_result();
    res->n = ix->n;
    res->stream = st;
    hj_status rs = dalloc(&res->table, ix->n, st);
    if (rs != HJ_OK) { delete res; return rs; }
    HJ_CUDA(cudaMemsetAsync(res->table, 0, (size_t)ix->n * sizeof(hj_nt_entry), st));
    const uint32_t key_bits = bits_for(ix->n);

    auto t_ref = std::chrono::steady_clock::now();
    float ms_group = 0;
    hj_status status = HJ_OK;
    while (!batches.empty()) {
        Batch b = batches.back();
        batches.pop_back();
        if (opts.max_batches && res->vals.size() >= opts.max_batches) {
            set_error("hj_join: batch limit %u reached", opts.max_batches);
            status = HJ_ERR_OVERFLOW;
            break;
        }
        HJ_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st));
        HJ_CUDA(cudaMemsetAsync(counters + 4, 0, sizeof(unsigned long long), st));
        HJ_CUDA(cudaMemsetAsync(overflow, 0, sizeof(uint32_t), st));
        PairSink sink{keys, vals, counters, cap, overflow};
        PairSink band = tc ? PairSink{band_q, band_c, counters + 4, cap, overflow} : no_band;
        status = run_refine(blocks + b.b0, b.b1 - b.b0, sink, band, 0, nullptr);
        if (status != HJ_OK) break;
        if (tc) {
            status = launch_band_recheck(ix, band_q, band_c, counters + 4, cap, sink, st);
            if (status != HJ_OK) break;
            status = check_timeout();
            if (status != HJ_OK) break;
        }
        unsigned long long used = 0;
        uint32_t ovf = 0;
        HJ_CUDA(cudaMemcpyAsync(&used, counters, 8, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaMemcpyAsync(&ovf, overflow, 4, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        if (ovf) {
            if (b.b1 - b.b0 <= 1) {
                set_error("hj_join: one work item produces more pairs than the result buffer holds (%llu)",
                          (unsigned long long)cap);
                status = HJ_ERR_OVERFLOW;
                break;
            }
            uint32_t mid = b.b0 + (b.b1 - b.b0) / 2;
            batches.push_back({mid, b.b1});
            batches.push_back({b.b0, mid});
            S.n_retries++;
            continue;
        }
        auto t_g = std::chrono::steady_clock::now();
        uint64_t slots = std::min<uint64_t>(used, cap);
        status = radix_sort_u32_u32(keys, vals, keys_tmp, vals_tmp, slots, key_bits, st);
        if (status != HJ_OK) break;
        unsigned long long valid = 0;
        if (slots) {
            k_count_valid<<<(unsigned)((slots + 255) / 256), 256, 0, st>>>(keys, slots, counters + 1);
            HJ_LAUNCHED();
            HJ_CUDA(cudaMemcpyAsync(&valid, counters + 1, 8, cudaMemcpyDeviceToHost, st));
            HJ_CUDA(cudaStreamSynchronize(st));
        }
        uint32_t bi = (uint32_t)res->vals.size();
        uint32_t* bv = nullptr;
        status = dalloc(&bv, valid, st);
        if (status != HJ_OK) break;
        if (valid) HJ_CUDA(cudaMemcpyAsync(bv, vals, valid * 4, cudaMemcpyDeviceToDevice, st));
        res->vals.push_back(bv);
        res->counts.push_back(valid);
        if (opts.keep_keys) {
            uint32_t* bk = nullptr;
            status = dalloc(&bk, valid, st);
            if (status != HJ_OK) break;
            if (valid) HJ_CUDA(cudaMemcpyAsync(bk, keys, valid * 4, cudaMemcpyDeviceToDevice, st));
            res->keys.push_back(bk);
        }
        if (valid) {
            k_table<<<(unsigned)((valid + 255) / 256), 256, 0, st>>>(keys, valid, bi, res->table);
            HJ_LAUNCHED();
        }
        res->total += valid;
        ms_group += ms_since(t_g);
    }
    HJ_CUDA(cudaStreamSynchronize(st));
    S.ms_refine = ms_since(t_ref) - ms_group;
    S.ms_group = ms_group;
    for (auto& ev : kev) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess) S.ms_refine_kernel += ms;
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
        S.refine_launches++;
    }
    cudaGetLastError();
    if (tc) {
        unsigned long long tcs[2] = {0, 0};
        HJ_CUDA(cudaMemcpyAsync(tcs, counters + 2, sizeof(tcs), cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        S.tc_accepts = tcs[0];
        S.band_pairs = tcs[1];
    }
    dfree(keys, st); dfree(vals, st); dfree(keys_tmp, st); dfree(vals_tmp, st);
    dfree(band_q, st); dfree(band_c, st);
    dfree(blocks, st); dfree(head, st); dfree(counters, st); dfree(flags, st);
    if (status == HJ_OK && !res->vals.empty()) {
        hj_status s2 = dalloc(&res->d_batch_vals, res->vals.size(), st);
        if (s2 == HJ_OK)
            s2 = cudaMemcpyAsync(res->d_batch_vals, res->vals.data(), res->vals.size() * sizeof(uint32_t*),
                                 cudaMemcpyHostToDevice, st) == cudaSuccess ? HJ_OK : HJ_ERR_CUDA;
        status = s2;
    }
    cudaStreamSynchronize(st);
    if (status != HJ_OK) {
        hj_result_destroy(res);
        return status;
    }
    S.total_pairs = res->total;
    S.n_batches = (uint32_t)res->vals.size();
    S.ms_total = ms_since(t_start);
    S.kernel_launches = (uint32_t)(thread_launch_count() - launches0);
    if (stats) *stats = S;
    *out = res;
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
