// hj_refine_plain.cu -- exact refine on the CUDA cores.
//
// Reference counterpart: kernelNDGridIndexGlobal (kernel.cu:727-802) with
// evaluateCell (kernel.cu:378-412) and evalPoint (kernel.cu:333-370), and the
// estimator kernel kernelNDGridIndexBatchEstimator_v2 (kernel.cu:607-716),
// which is this kernel in count-only mode.
//
// Semantics kept bit for bit: a pair (q, c) is emitted iff c lies in one of
// the non-empty cells of q's 3^k stencil (unsigned clamp with the wrap at
// coordinate 0, kernel.cu:780-781) and
//     acc = 0; for l in 0..d-1: diff = c_l - q_l; acc = fma(diff, diff, acc)
// satisfies sqrt(acc) <= eps, evaluated as acc <= thr where thr is the largest
// value of the dataset type whose correctly rounded sqrt is <= eps.
//
// B200 design: a persistent grid pulls work items (up to QB queries of one
// cell) from the workload-ordered block list with one atomic per item.  The
// cell's stencil is resolved once per item into contiguous point ranges
// (rows of the stencil along dimension 0), the candidates are streamed through
// shared memory in chunks of CB points (transposed to dimension-major), and
// each thread evaluates an RQ x RC register tile of (query, candidate) pairs.
// Hits are appended with warp-aggregated reservations into the pair sink.

#include <algorithm>
#include <atomic>
#include <type_traits>

#include "hj_internal.h"

namespace hj {
namespace {

constexpr uint32_t kRowGroup = 256;   // stencil rows resolved per pass
constexpr uint32_t kNoPos = 0xFFFFFFFFu;

template <typename T>
struct PlainArgs {
    const T* pts;
    const uint32_t* perm;
    const unsigned long long* cell_lid;
    const uint32_t* cell_start;
    uint32_t nC;
    HjCellHash hash;
    uint32_t d;
    HjGrid grid;
    T thr;
    const HjBlock* blocks;
    uint32_t nblocks;
    unsigned int* head;
    PairSink sink;
    uint32_t count_only;
    unsigned long long* block_counts;   // count-only mode: pairs per work item
    uint32_t* qcount;                   // optional: pairs per query (original id), written by the block
                                        // path's items where plain_counts_queries() holds; zeroed by the caller
};

// Dimension classes whose refine counts each query's pairs (qcount): 2-D and 3-D,
// the low dimensions where pairs far outnumber the arithmetic (the counters cost
// registers that higher d needs).  Only without the warp path (k < 4) does every
// item take the block path that counts.
template <int D>
constexpr bool kCountsQueries = D == 2 || D == 3;


// Packed FP32 pairs (sm_100): each lane's result is the IEEE-rounded scalar
// operation, so the packed loop is bit-identical to the scalar one.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    return ((unsigned long long)__float_as_uint(hi) << 32) | __float_as_uint(lo);
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double ffma(double a, double b, double c) { return __fma_rn(a, b, c); }

// Warp path for small work items: one warp joins one item on its own, with no
// block-wide barrier.  The item's queries (at most 32 / D of them per pass) sit
// in lane registers and are broadcast with shuffles; every lane resolves its
// own stencil rows through the cell hash (RPL rows per round), and the round's
// row ranges are laid end to end: in each step the 32 lanes take 32 consecutive
// candidates of that concatenation (each lane following its own pointer through
// the ranges), so a round costs ceil(candidates / 32) steps however the
// candidates spread over its rows.
// Used once the workload order reaches items with nq * D <= 32 and at most
// 4096 candidate pairs, when k >= 4 (3^(k-1) >= 27 stencil rows per item):
// there the block path's barriers and staging cost more than the pairs.
constexpr uint32_t kWarpRPL = 4;

template <typename T, int D>
__device__ __forceinline__ void warp_item(const PlainArgs<T>& a, const HjBlock& blk, WarpChunk& wc, uint32_t* wsm,
                                          uint32_t* wrng, unsigned long long& item_cnt) {
    constexpr uint32_t G = 32u / D;      // queries per pass
    constexpr uint32_t RPL = kWarpRPL;   // stencil rows per lane per round
    const uint32_t lane = lane_id();
    const uint32_t k = a.grid.k;
    const uint32_t nq = blk.q1 - blk.q0;
    const unsigned long long L = a.cell_lid[blk.cell];
    uint32_t lo[kMaxK], w[kMaxK];
    uint32_t rows = 1;
    bool empty = false;
    const uint32_t cl = lane_cell_coord(a.grid, L);
    for (uint32_t j = 0; j < k; ++j) {
        const uint32_t c = __shfl_sync(0xffffffffu, cl, j);
        uint32_t l = c - 1u;                                // kernel.cu:780, wraps at 0
        uint32_t h = min(a.grid.n_cells[j] - 1u, c + 1u);   // kernel.cu:781
        empty |= l > h;
        lo[j] = l;
        w[j] = h - l + 1u;
        if (j > 0) rows *= w[j];
    }
    if (empty) return;
    const StencilRows sr = stencil_rows(a.grid, lo, rows);
    uint32_t* cid_w = wsm;        // [32] candidate ids of the current step
    uint32_t* qid_w = wsm + 32;   // [32] original ids of the current pass's queries
    for (uint32_t qg = 0; qg < nq; qg += G) {
        const uint32_t gq = min(G, nq - qg);
        // lane L holds coordinate L % D of query qg + L / D
        const T qv = lane < gq * D ? a.pts[(size_t)(blk.q0 + qg + lane / D) * D + lane % D] : T(0);
        if (!a.count_only) qid_w[lane] = lane < gq ? a.perm[blk.q0 + qg + lane] : 0u;
        __syncwarp();
        for (uint32_t rb = 0; rb < rows; rb += 32 * RPL) {
            uint32_t st[RPL], len[RPL];
#pragma unroll
            for (uint32_t sl = 0; sl < RPL; ++sl) {
                const uint32_t r = rb + sl * 32 + lane;
                st[sl] = 0;
                len[sl] = 0;
                if (r < rows) {
                    const uint2 sp = cell_span(a.hash, a.cell_start, stencil_row_id(a.grid, sr, lo, w, r), w[0]);
                    st[sl] = sp.x;
                    len[sl] = sp.y - sp.x;
                }
            }
            // the round's ranges end to end: range j = sl * 32 + lane starts at candidate
            // offset pre[j] of the concatenation (pre[32 * RPL] = the round's candidates)
            uint32_t* rst = wrng;                     // [32 * RPL] range starts (sorted positions)
            uint32_t* pre = wrng + 32 * RPL;          // [32 * RPL + 1] exclusive prefix of the lengths
            uint32_t run = 0;
#pragma unroll
            for (uint32_t sl = 0; sl < RPL; ++sl) {
                uint32_t incl = len[sl];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= (uint32_t)o) incl += t;
                }
                rst[sl * 32 + lane] = st[sl];
                pre[sl * 32 + lane] = run + incl - len[sl];
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) pre[32 * RPL] = run;
            __syncwarp();
            uint32_t j = 0;   // this lane's current range
            for (uint32_t base = 0; base < run; base += 32) {
                const uint32_t idx = base + lane;
                const bool valid = idx < run;
                while (j + 1 < 32 * RPL && pre[j + 1] <= idx) ++j;
                const uint32_t p = valid ? rst[j] + (idx - pre[j]) : 0u;
                T cv[D];
#pragma unroll
                for (int l = 0; l < D; ++l) cv[l] = valid ? a.pts[(size_t)p * D + l] : T(0);
                uint32_t mask = 0;
#pragma unroll
                for (uint32_t qi = 0; qi < G; ++qi) {
                    T acc = T(0);
#pragma unroll
                    for (int l = 0; l < D; ++l) {
                        const T q = __shfl_sync(0xffffffffu, qv, qi * D + l);
                        const T diff = fsub(cv[l], q);   // candidate - query (kernel.cu:351)
                        acc = ffma(diff, diff, acc);
                    }
                    mask |= (uint32_t)(valid && qi < gq && acc <= a.thr) << qi;
                }
                if (a.count_only) {
                    item_cnt += __popc(mask);
                } else {
                    cid_w[lane] = valid ? a.perm[p] : 0u;
                    __syncwarp();
                    warp_emit_masks(a.sink, wc, mask,
                                    [&](uint32_t owner, uint32_t b) { return make_uint2(qid_w[b], cid_w[owner]); });
                    __syncwarp();
                }
            }
            __syncwarp();   // the next round rewrites the ranges
        }
        __syncwarp();
    }
}

template <typename T, int D, int QB, int CB, int RQ, int RC>
__global__ void __launch_bounds__(256, 3) k_refine_plain(PlainArgs<T> a) {
    static_assert((QB / RQ) * (CB / RC) == 256, "tile must map onto 256 threads");
    static_assert(RQ * RC <= 32, "hit mask is 32 bits");
    constexpr int TX = CB / RC;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t d = D ? (uint32_t)D : a.d;
    T* q_s = reinterpret_cast<T*>(smem);                        // [d][QB]
    T* c_s = q_s + (size_t)d * QB;                              // [d][CB]
    uint32_t* qid_s = reinterpret_cast<uint32_t*>(c_s + (size_t)d * CB);  // [QB]
    uint32_t* cpos_s = qid_s + QB;                              // [CB]
    uint32_t* cid_s = cpos_s + CB;                              // [CB] original ids of the chunk
    uint32_t* rs = cid_s + CB;                                  // [kRowGroup] range starts
    uint32_t* rp = rs + kRowGroup;                              // [kRowGroup + 1] prefix of lengths
    __shared__ uint32_t s_item;
    __shared__ uint32_t wsum_s[17];   // row-group scan: warp totals, their prefixes, the group total
    __shared__ uint32_t warp_sm[8][64];   // warp path: candidate and query ids per warp
    __shared__ uint32_t warp_rng[8][2 * 32 * kWarpRPL + 1];   // warp path: a round's row ranges per warp
    constexpr bool kWarpPath = D != 0 && D <= 32;

    const uint32_t tid = threadIdx.x;
    const uint32_t tx = tid % TX, ty = tid / TX;
    const uint32_t k = a.grid.k;
    WarpChunk wc;
    warp_chunk_init(wc);

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.head, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= a.nblocks) break;
        const HjBlock blk = a.blocks[item];
        const uint32_t nq = blk.q1 - blk.q0;

        if constexpr (kWarpPath) {
            // from the first item whose queries fit the warp path, every warp of the block
            // takes items on its own until the order is exhausted (the decision is
            // block-uniform: all threads read the same item)
            if (k >= 4u && nq * (uint32_t)D <= 32u && (unsigned long long)blk.nb * nq <= 4096ull) {
                const uint32_t wid = tid >> 5;
                uint32_t it_w = item;   // warp 0 takes the item already fetched
                if (wid != 0) {
                    uint32_t nx = 0;
                    if (lane_id() == 0) nx = atomicAdd(a.head, 1u);
                    it_w = __shfl_sync(0xffffffffu, nx, 0);
                }
                while (it_w < a.nblocks) {
                    unsigned long long cnt_w = 0;
                    warp_item<T, D>(a, a.blocks[it_w], wc, warp_sm[wid], warp_rng[wid], cnt_w);
                    if (a.count_only) {
                        for (int o = 16; o > 0; o >>= 1) cnt_w += __shfl_down_sync(0xffffffffu, cnt_w, o);
                        if (lane_id() == 0 && cnt_w) atomicAdd(&a.block_counts[it_w], cnt_w);
                    }
                    uint32_t nx = 0;
                    if (lane_id() == 0) nx = atomicAdd(a.head, 1u);
                    it_w = __shfl_sync(0xffffffffu, nx, 0);
                }
                break;
            }
        }

        // queries, dimension-major
        for (uint32_t f = tid; f < (uint32_t)QB * d; f += 256) {
            uint32_t i = f / d, l = f - i * d;
            q_s[l * QB + i] = i < nq ? a.pts[(size_t)(blk.q0 + i) * d + l] : T(0);
        }
        for (uint32_t i = tid; i < (uint32_t)QB; i += 256) qid_s[i] = i < nq ? a.perm[blk.q0 + i] : 0u;

        // stencil box from the cell's linear id (its digits are every member's coordinates)
        const unsigned long long L = a.cell_lid[blk.cell];
        uint32_t lo[kMaxK], w[kMaxK];
        uint32_t rows = 1;
        bool empty = false;
        const uint32_t cl = lane_cell_coord(a.grid, L);
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t c = __shfl_sync(0xffffffffu, cl, j);
            uint32_t l = c - 1u;                                // kernel.cu:780, wraps at 0
            uint32_t h = min(a.grid.n_cells[j] - 1u, c + 1u);   // kernel.cu:781
            empty |= l > h;
            lo[j] = l;
            w[j] = h - l + 1u;
            if (j > 0) rows *= w[j];
        }
        unsigned long long item_cnt = 0;
        uint32_t qc[RQ];   // this thread's pairs per query of its tile rows (qcount)
#pragma unroll
        for (int r = 0; r < RQ; ++r) qc[r] = 0;
        if (!empty) {
            for (uint32_t row0 = 0; row0 < rows; row0 += kRowGroup) {
                const uint32_t nr = min(kRowGroup, rows - row0);
                __syncthreads();
                {
                    // every thread resolves one row of this group into a point range (through
                    // the cell hash), then the block prefixes the lengths: warp scans, then a
                    // scan of the 8 warp totals
                    uint32_t len = 0;
                    if (tid < nr) {
                        const StencilRows sr = stencil_rows(a.grid, lo, rows);   // not kept across the item
                        const uint2 sp =
                            cell_span(a.hash, a.cell_start, stencil_row_id(a.grid, sr, lo, w, row0 + tid), w[0]);
                        rs[tid] = sp.x;
                        len = sp.y - sp.x;
                    }
                    uint32_t incl = len;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane_id() >= (uint32_t)o) incl += t;
                    }
                    if (lane_id() == 31) wsum_s[tid >> 5] = incl;
                    __syncthreads();
                    if (tid < 32) {
                        uint32_t v = tid < 8 ? wsum_s[tid] : 0u, x = v;
#pragma unroll
                        for (int o = 1; o < 8; o <<= 1) {
                            uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
                            if (tid >= (uint32_t)o) x += t;
                        }
                        if (tid < 8) wsum_s[8 + tid] = x - v;   // exclusive warp offsets
                        if (tid == 7) wsum_s[16] = x;           // group total
                    }
                    __syncthreads();
                    if (tid < nr) rp[tid] = wsum_s[8 + (tid >> 5)] + incl - len;
                    if (tid == 0) rp[nr] = wsum_s[16];
                }
                __syncthreads();
                const uint32_t total = rp[nr];
                for (uint32_t cb = 0; cb < total; cb += CB) {
                    for (uint32_t j = tid; j < (uint32_t)CB; j += 256) {
                        uint32_t v = cb + j, p = kNoPos;
                        if (v < total) {
                            uint32_t lo2 = 0, hi2 = nr;   // last r with rp[r] <= v
                            while (hi2 - lo2 > 1) {
                                uint32_t mid = (lo2 + hi2) >> 1;
                                if (rp[mid] <= v) lo2 = mid; else hi2 = mid;
                            }
                            p = rs[lo2] + (v - rp[lo2]);
                        }
                        cpos_s[j] = p;
                        // staged once per chunk, so emitting a pair reads shared memory only
                        if (!a.count_only) cid_s[j] = p != kNoPos ? a.perm[p] : 0u;
                    }
                    __syncthreads();
                    for (uint32_t f = tid; f < (uint32_t)CB * d; f += 256) {
                        uint32_t l = f / CB, j = f - l * CB;
                        uint32_t p = cpos_s[j];
                        c_s[f] = p != kNoPos ? a.pts[(size_t)p * d + l] : T(0);
                    }
                    __syncthreads();
                    const uint32_t nvalid = min((uint32_t)CB, total - cb);
                    // threads whose whole tile lies past the queries or the candidates skip the
                    // arithmetic (small work items: one query against a few candidates)
                    const bool live = ty * RQ < nq && tx * RC < nvalid;

                    T acc[RQ][RC];
                    if (!live) {
#pragma unroll
                        for (int r = 0; r < RQ; ++r)
#pragma unroll
                            for (int c = 0; c < RC; ++c) acc[r][c] = T(0);
                    } else if constexpr (std::is_same<T, float>::value && RC % 2 == 0) {
                        // candidate pairs (c, c+1) packed: diff = c - q, acc = fma(diff, diff, acc)
                        unsigned long long acc2[RQ][RC / 2];
#pragma unroll
                        for (int r = 0; r < RQ; ++r)
#pragma unroll
                            for (int c = 0; c < RC / 2; ++c) acc2[r][c] = 0ull;
#pragma unroll(D ? (D <= 8 ? D : 6) : 1)
                        for (uint32_t l = 0; l < d; ++l) {
                            unsigned long long cv2[RC / 2];
                            const unsigned long long* cp =
                                reinterpret_cast<const unsigned long long*>(&c_s[l * CB + tx * RC]);
#pragma unroll
                            for (int c = 0; c < RC / 2; ++c) cv2[c] = cp[c];
#pragma unroll
                            for (int r = 0; r < RQ; ++r) {
                                const float q = q_s[l * QB + ty * RQ + r];
                                const unsigned long long qq = pack2(q, q);
#pragma unroll
                                for (int c = 0; c < RC / 2; ++c) {
                                    unsigned long long diff = sub2(cv2[c], qq);   // candidate - query (kernel.cu:351)
                                    acc2[r][c] = fma2(diff, diff, acc2[r][c]);
                                }
                            }
                        }
#pragma unroll
                        for (int r = 0; r < RQ; ++r)
#pragma unroll
                            for (int c = 0; c < RC / 2; ++c) {
                                acc[r][2 * c] = __uint_as_float((uint32_t)acc2[r][c]);
                                acc[r][2 * c + 1] = __uint_as_float((uint32_t)(acc2[r][c] >> 32));
                            }
                    } else {
#pragma unroll
                        for (int r = 0; r < RQ; ++r)
#pragma unroll
                            for (int c = 0; c < RC; ++c) acc[r][c] = T(0);
#pragma unroll(D ? (D <= 8 ? D : 6) : 1)
                        for (uint32_t l = 0; l < d; ++l) {
                            T qv[RQ], cv[RC];
#pragma unroll
                            for (int r = 0; r < RQ; ++r) qv[r] = q_s[l * QB + ty * RQ + r];
#pragma unroll
                            for (int c = 0; c < RC; ++c) cv[c] = c_s[l * CB + tx * RC + c];
#pragma unroll
                            for (int r = 0; r < RQ; ++r)
#pragma unroll
                                for (int c = 0; c < RC; ++c) {
                                    T diff = fsub(cv[c], qv[r]);          // candidate - query (kernel.cu:351)
                                    acc[r][c] = ffma(diff, diff, acc[r][c]);
                                }
                        }
                    }
                    uint32_t mask = 0;
#pragma unroll
                    for (int r = 0; r < RQ; ++r)
#pragma unroll
                        for (int c = 0; c < RC; ++c) {
                            bool hit = live && acc[r][c] <= a.thr && (ty * RQ + r) < nq && (tx * RC + c) < nvalid;
                            mask |= (hit ? 1u : 0u) << (r * RC + c);
                        }
                    if (a.count_only) {
                        item_cnt += __popc(mask);
                    } else {
                        if constexpr (kCountsQueries<D>) {
                            if (a.qcount) {
#pragma unroll
                                for (int r = 0; r < RQ; ++r) qc[r] += __popc((mask >> (r * RC)) & ((1u << RC) - 1u));
                            }
                        }
                        // coalesced output: each lane writes every 32nd pair of the warp's hits
                        const uint32_t wbase = tid & ~31u;
                        warp_emit_masks(a.sink, wc, mask, [&](uint32_t owner, uint32_t b) {
                            const uint32_t ot = wbase + owner;
                            const uint32_t qi = (ot / TX) * RQ + b / RC, cj = (ot % TX) * RC + b % RC;
                            return make_uint2(qid_s[qi], cid_s[cj]);
                        });
                    }
                    __syncthreads();
                }
            }
        }
        if (a.count_only) {
            for (int o = 16; o > 0; o >>= 1) item_cnt += __shfl_down_sync(0xffffffffu, item_cnt, o);
            if (lane_id() == 0 && item_cnt) atomicAdd(&a.block_counts[item], item_cnt);
        } else if constexpr (kCountsQueries<D>) {
            if (a.qcount) {
                // the TX threads of a tile row share its RQ queries: sum over them, one store
                // per query (a query belongs to one item of a batch)
                static_assert(TX <= 32 && (32 % TX) == 0, "tile rows within a warp");
#pragma unroll
                for (int r = 0; r < RQ; ++r) {
                    uint32_t v = qc[r];
#pragma unroll
                    for (int o = TX / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    const uint32_t qi = ty * RQ + r;
                    if (tx == 0 && qi < nq && v) a.qcount[qid_s[qi]] = v;
                }
            }
        }
        __syncthreads();
    }
    if (!a.count_only) warp_chunk_close(a.sink, wc);
}

template <typename T, int D, int QB, int CB, int RQ, int RC>
hj_status launch_t(const PlainArgs<T>& args, cudaStream_t st) {
    size_t smem = (size_t)(D ? D : args.d) * (QB + CB) * sizeof(T) + (QB + 2 * CB + 2 * kRowGroup + 1) * sizeof(uint32_t);
    auto kern = k_refine_plain<T, D, QB, CB, RQ, RC>;
    HJ_TRY(ensure_smem(kern, smem));
    // resident blocks per SM, queried once per kernel and shared-memory size (a driver call)
    static std::atomic<int> s_per_sm{0};
    static std::atomic<size_t> s_smem{0};
    int per_sm = s_per_sm.load(std::memory_order_relaxed);
    if (per_sm == 0 || s_smem.load(std::memory_order_relaxed) != smem) {
        HJ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
        s_smem.store(smem, std::memory_order_relaxed);
        s_per_sm.store(per_sm, std::memory_order_relaxed);
    }
    if (per_sm < 1) {
        set_error("refine: %zu bytes of shared memory per block do not fit", smem);
        return HJ_ERR_UNSUPPORTED;
    }
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)per_sm * num_sms(), std::max<uint32_t>(args.nblocks, 1));
    kern<<<grid, 256, smem, st>>>(args);
    HJ_LAUNCHED();
    return HJ_OK;
}

// Two tile shapes per dimension class, both with 64-query work items and 256
// threads: 64 queries x 128 candidates per staged chunk (4 x 8 per thread) and
// 64 x 64 (4 x 4 per thread).  The wide one stages half as many chunks (half
// the barriers) but holds twice the accumulators; which wins depends on d, the
// type and the hit density, so the join times both on the estimator's sample
// (shape 0 is each type's default: wide for float, narrow for double).
template <typename T, int D>
hj_status launch_shape(const PlainArgs<T>& a, int wide, cudaStream_t st) {
    return wide ? launch_t<T, D, 64, 128, 4, 8>(a, st) : launch_t<T, D, 64, 64, 4, 4>(a, st);
}

template <typename T>
hj_status dispatch_t(const PlainArgs<T>& args, int shape, cudaStream_t st);

template <>
hj_status dispatch_t<float>(const PlainArgs<float>& a, int shape, cudaStream_t st) {
    const int wide = shape == 0;
    switch (a.d) {
        case 2: return launch_shape<float, 2>(a, wide, st);
        case 3: return launch_shape<float, 3>(a, wide, st);
        case 6: return launch_shape<float, 6>(a, wide, st);
        case 18: return launch_shape<float, 18>(a, wide, st);
        case 32: return launch_shape<float, 32>(a, wide, st);
        case 90: return launch_shape<float, 90>(a, wide, st);
        default: return launch_shape<float, 0>(a, wide, st);
    }
}
template <>
hj_status dispatch_t<double>(const PlainArgs<double>& a, int shape, cudaStream_t st) {
    const int wide = shape != 0;
    switch (a.d) {
        case 2: return launch_shape<double, 2>(a, wide, st);
        case 3: return launch_shape<double, 3>(a, wide, st);
        case 6: return launch_shape<double, 6>(a, wide, st);
        default: return launch_shape<double, 0>(a, wide, st);
    }
}

}  // namespace

uint32_t plain_query_block(int dtype) { return 64; (void)dtype; }

// Whether the exact refine writes each query's pair count (PlainArgs::qcount) for
// this index: a counting dimension class, and every item on the block path.
bool plain_counts_queries(const hj_index* ix) { return ix->grid.k < 4 && (ix->d == 2 || ix->d == 3); }

// Upper bound on the warps of one refine launch that reserve pair-sink chunks (each
// holds at most one partly filled chunk): at most 8 blocks of 8 warps per SM, and
// never more blocks than work items.
uint64_t plain_emit_warps(uint32_t nblocks) {
    return (uint64_t)std::min<uint64_t>(8ull * num_sms(), std::max<uint32_t>(nblocks, 1)) * 8ull;
}

// Runs the exact refine over work items blocks[0..nblocks).  `head` must be
// zero on entry.  count_only: per-item pair counts go to block_counts.
hj_status launch_refine_plain(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                              const PairSink& sink, uint32_t count_only, unsigned long long* block_counts,
                              uint32_t* qcount, cudaStream_t st) {
    if (nblocks == 0) return HJ_OK;
    if (ix->dtype == HJ_F32) {
        PlainArgs<float> a{(const float*)ix->pts, ix->perm, ix->cell_lid, ix->cell_start, ix->nC, cell_hash(ix), ix->d,
                           ix->grid,
                           (float)ix->thr, blocks, nblocks, head, sink, count_only, block_counts, qcount};
        return dispatch_t<float>(a, ix->plain_shape, st);
    }
    PlainArgs<double> a{(const double*)ix->pts, ix->perm, ix->cell_lid, ix->cell_start, ix->nC, cell_hash(ix), ix->d,
                        ix->grid,
                        ix->thr, blocks, nblocks, head, sink, count_only, block_counts, qcount};
    return dispatch_t<double>(a, ix->plain_shape, st);
}

}  // namespace hj
