// hj_refine_tc.cu -- tensor-core squared-distance filter with exact recheck.
//
// Reference counterpart: the refine kernelNDGridIndexGlobal (kernel.cu:727-802,
// evalPoint kernel.cu:333-370).  For high dimensions the reference's candidate
// loop is a dense distance evaluation; here each (candidate tile x query block)
// is a GEMM on the 5th-generation tensor cores:
//
//   A (M = 128 candidates, streamed by TMA) = [-2 c~, 1, 1, |c~|^2_hi, |c~|^2_lo, 0...]
//   B (N = 2 x 256 queries, resident)       = [  q~, |q~|^2_hi, |q~|^2_lo, 1, 1, 0...]
//   D = A B^T = |q~|^2 + |c~|^2 - 2 q~.c~ = |q~ - c~|^2        (FP32 accumulate in TMEM)
//
// where x~ is the FP16 (or BF16) rounding of (x - origin) * 2^s.  The origin
// is the per-dimension minimum and s is a power-of-two scale chosen per
// dataset so that the largest |x - origin|^2 * 4^s lies in [2^12, 2^14]: every
// stored half (coordinates up to 128, -2x up to 256, norm halves up to 2^14)
// is finite with a 4x margin below FP16's 65504 whatever the data's units, and
// small-valued data stays clear of the FP16 subnormals.  Scaling by 2^s is
// exact, so the threshold becomes T * 4^s exactly.  The norms ride in the K
// padding (d + 4 rounded up to 32), so the MMA yields the (scaled) squared
// distance directly and the epilogue is one compare per pair.  A pair is
//   accepted  if D <= T - delta,
//   rejected  if D >  T + delta,
//   rechecked otherwise, in FP32 in the reference's order (fma chain),
// with T the exact squared threshold and delta a per-candidate-row bound on
// |D - d2_ref| (quantisation error, norm-split residual, tensor-core
// accumulation error and the reference's own FP32 rounding; derivation in
// tc_band_p / tc_band_q below).  A D that is NaN counts as "in the band", never as a
// reject.  The result set is therefore identical to the exact path.
//
// Kernel shape (one CTA per SM, persistent, 96 + 128 * EPI threads):
//   warp 0      TMA producer: the work item's 256 queries once, candidate tiles
//               through a ring of shared-memory stages;
//   warps 1, 2  MMA issuers: candidate tile t is computed as M = 128 x N = 256
//               MMAs into TMEM accumulator t % 2 (2 x 256 columns, all of TMEM)
//               by issuer 1 + t % 2.  The accumulators form a ring over the
//               tiles, so the MMAs of tile t + 1 run while the epilogue drains
//               tile t.  N = 256 matters: a microbenchmark of this pattern
//               issued 128 x 128 x 16 MMAs at 42% of the tensor pipe's rate and
//               128 x 256 x 16 ones at 98%;
//   warps 3..   epilogue, EPI groups of 4 warps (one per TMEM lane quarter),
//               either all draining every tile or split into one set per
//               accumulator (every other tile; autotuned): tcgen05.ld,
//               min-reduce, compare, warp-aggregated emission; an accumulator
//               is released as soon as its warps have read it.
// Every wait is bounded; a timeout raises an error flag, drains and returns.

#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "hj_internal.h"
#include "hj_tc.cuh"

namespace hj {
namespace {

constexpr int kQT = 2;                       // 128-row query loads per work item
constexpr int kTileRows = 128;               // rows per tile (M for A) and per query load
constexpr int kQB = kQT * kTileRows;         // queries per work item (N of every MMA)
constexpr int kAcc = 2;                      // TMEM accumulators: a ring over the candidate tiles
constexpr int kAccCols = 256;                // N of one MMA: the work item's queries
constexpr int kProbeThreads = 192;   // tile probe: TMA warp, MMA warp, 4 epilogue warps
constexpr int kProbeQT = 4;                  // the tile probe evaluates 512 query rows ...
constexpr int kProbeQB = kProbeQT * kTileRows;
constexpr int kMaxStages = 8;
constexpr uint32_t kKBlockBytes = kTileRows * 64;   // one 32-element K block of a 128-row tile
constexpr uint32_t kBKBlockBytes = kQB * 64;        // one 32-element K block of the whole query block
constexpr uint32_t kProbeBKBlockBytes = kProbeQB * 64;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kMaxRanges = 256;
constexpr long long kWaitCycles = 4000000000ll;     // ~2 s at 1.9 GHz

struct TcArgs {
    const HjBlock* blocks;
    uint32_t nblocks;
    unsigned int* head;
    const uint32_t* perm;
    const unsigned long long* cell_lid;
    const uint32_t* cell_start;
    uint32_t nC;
    HjCellHash hash;
    HjGrid grid;
    const float4* pinfo;        // per sorted point: quantisation error norm, |x~|^2, norm-split residual
    const float* pband;         // per sorted point: its part of the guard band (tc_band_p)
    uint32_t n;
    uint32_t nkb;               // K blocks of 32 elements
    uint32_t stages;
    float thr;
    float gamma_acc;
    float s_t;                  // sqrt(T (1 + 1e-4))
    float ref_rel;              // (d + 2) 2^-24 (1.01)
    PairSink sink;              // accepted pairs: (query id, candidate id)
    PairSink band;              // band pairs: (query sorted position, candidate sorted position)
    uint32_t count_only;
    unsigned long long* block_counts;
    unsigned long long* stats;  // [0] accepted, [1] band
    uint32_t* err;
    uint32_t idesc;
    long long wait_cycles;      // bound of every mbarrier wait (SM cycles)
};

struct TcShared {
    uint64_t full_a[kMaxStages];
    uint64_t empty_a[kMaxStages];
    uint64_t full_acc[kAcc];
    uint64_t empty_acc[kAcc];
    uint64_t bfull;
    uint32_t tmem_base;
    uint32_t item;
    uint32_t abort;
    uint32_t nq, ntiles, nr, q0;
    uint32_t max_e, max_n, max_r;          // float bits (non-negative)
    uint32_t qid[kQB];
    uint32_t rs[kMaxRanges];               // range start (sorted position)
    uint32_t rl[kMaxRanges];               // range length
    uint32_t tp[kMaxRanges + 1];           // tile prefix
};


// Tiles are visited in order, so the range of tile t is found by walking r
// forward from the previous tile's range (the last r with tp[r] <= t; ranges
// without tiles are stepped over) instead of a binary search per tile.  The
// current range's first tile, end tile, start row and length stay in registers,
// so a tile inside the same range costs no shared-memory reads.
struct TileWalk {
    uint32_t r = 0, start = 0, valid = 0;
    uint32_t t0 = 0, t1 = 0, rs = 0, rl = 0;   // range r: tiles [t0, t1), rows [rs, rs + rl)
    __device__ __forceinline__ void locate(const TcShared& S, uint32_t t) {
        if (t >= t1) {
            while (r + 1 < S.nr && S.tp[r + 1] <= t) ++r;
            t0 = S.tp[r];
            t1 = r + 1 < S.nr ? S.tp[r + 1] : 0xFFFFFFFFu;
            rs = S.rs[r];
            rl = S.rl[r];
        }
        const uint32_t off = (t - t0) * kTileRows;
        start = rs + off;
        valid = min((uint32_t)kTileRows, rl - off);
    }
};

// The guard band of a candidate row c against the whole query block:
//   |D - d2_ref| <= acc + res + e (2 sT + 3 e) + ref_rel (sT + e)^2
//   e   = e_c + max e_q       (|x~ - x| norms; |(|q~-c~|) - |q-c|| <= e)
//   acc = gamma (2.01 (|c~|^2 + max |q~|^2))   (tensor-core accumulation; 2|a.b| <= |a|^2 + |b|^2)
//   res = r_c + max r_q       (norm split residuals)
//   the last term bounds the reference's own FP32 rounding of d2 (d + 2 roundings).
// With (e_c + m)^2 <= 2 e_c^2 + 2 m^2 it splits into a candidate part and a
// query-block part, delta <= P(c) + Q(block):
//   P(c) = gamma 2.01 |c~|^2 + r_c + e_c (2 sT + 6 e_c) + ref_rel (2 sT e_c + 2 e_c^2)
//   Q    = gamma 2.01 max|q~|^2 + max r_q + m (2 sT + 6 m) + ref_rel (sT^2 + 2 sT m + 2 m^2),  m = max e_q
// each with a 1% margin for its own FP32 evaluation.  P is computed once per
// point (k_tc_pband, rounded up), Q once per work item, and a row's band edges
// are two additions rounded outwards: hi = (thr + Q) + P, lo = (thr - Q) - P.
__host__ __device__ __forceinline__ double tc_band_p(double gamma, double s_t, double ref_rel, double e, double n2,
                                                     double r) {
    return (gamma * 2.01 * n2 + r + e * (2.0 * s_t + 6.0 * e) + ref_rel * (2.0 * s_t * e + 2.0 * e * e)) * 1.01;
}
__host__ __device__ __forceinline__ double tc_band_q(double gamma, double s_t, double ref_rel, double me, double mn,
                                                     double mr) {
    return (gamma * 2.01 * mn + mr + me * (2.0 * s_t + 6.0 * me) +
            ref_rel * (s_t * s_t + 2.0 * s_t * me + 2.0 * me * me)) * 1.01 + 1e-30;
}

// Tree minimum of N values with three-input minima.  The .NaN forms return NaN
// when any input is NaN, so a NaN accumulator reaches the band test below
// (where "not above the upper edge" counts it as a hit) instead of being
// dropped by the minimum.
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.NaN.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin2(float a, float b) {
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
// A value is a candidate hit unless it is known to lie above the band: NaN is
// kept (and, failing `v <= lo`, goes to the exact recheck).
__device__ __forceinline__ bool not_above(float v, float hi) { return !(v > hi); }
template <uint32_t N>
__device__ __forceinline__ float minN(const float (&v)[N]) {
    if constexpr (N == 1) {
        return v[0];
    } else if constexpr (N == 2) {
        return fmin2(v[0], v[1]);
    } else {
        constexpr uint32_t M = (N + 2) / 3;
        float m[M];
#pragma unroll
        for (uint32_t i = 0; i < N / 3; ++i) m[i] = fmin3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        if constexpr (N % 3 == 1) m[M - 1] = v[N - 1];
        if constexpr (N % 3 == 2) m[M - 1] = fmin2(v[N - 2], v[N - 1]);
        return minN<M>(m);
    }
}

// EPI = epilogue warp groups (4 warps each, one per TMEM lane quarter).  SPLIT:
// the epilogue warps form one set per accumulator, so a warp drains every other
// tile (with two tiles' MMA time for it) instead of every tile.  Which is faster
// depends on d: the autotuner times all four shapes.  DEFER: one vote per
// accumulator instead of one per chunk, chunks with a hit read again before the
// release; it pays where hits are rare (picked from the estimated pair density).
template <int EPI, bool SPLIT, bool DEFER>
__global__ void __launch_bounds__(32 * (1 + kAcc) + 128 * EPI, 1)
    k_refine_tc(const __grid_constant__ CUtensorMap tm_cand, const __grid_constant__ CUtensorMap tm_query, TcArgs a) {
    static_assert(EPI == 2 || EPI == 4, "an epilogue set needs whole groups of 4 warps");
    extern __shared__ uint8_t smem_raw[];
    // operand tiles need 1024-byte alignment for the swizzle pattern
    uint32_t base = tc::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    const uint32_t tile_bytes = a.nkb * kKBlockBytes;
    uint8_t* b_tiles = smem;                                   // query block: [K block][256 rows]
    uint8_t* a_tiles = smem + kQT * tile_bytes;                // a.stages tiles: [K block][128 rows]
    TcShared& S = *reinterpret_cast<TcShared*>(a_tiles + a.stages * tile_bytes);

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    if (tid == 0) {
        for (uint32_t s = 0; s < a.stages; ++s) {
            tc::mbar_init(&S.full_a[s], 1);
            tc::mbar_init(&S.empty_a[s], 1);   // released by the one issuer of the tile it holds
        }
        for (int j = 0; j < kAcc; ++j) {
            tc::mbar_init(&S.full_acc[j], 1);
            tc::mbar_init(&S.empty_acc[j], SPLIT ? 2 * EPI : 4 * EPI);   // the warps draining it
        }
        tc::mbar_init(&S.bfull, 1);
        S.abort = 0;
        tc::fence_mbar_init();
        tc::tma_prefetch_desc(&tm_cand);
        tc::tma_prefetch_desc(&tm_query);
    }
    if (warp == 1) {
        tc::tmem_alloc(&S.tmem_base, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = S.tmem_base;
    volatile uint32_t* abort = &S.abort;

    // role state carried across work items (barrier phases)
    uint32_t it = 0;            // candidate tiles issued / consumed
    uint32_t acc_use[kAcc] = {0, 0};   // uses of each accumulator seen by this thread
    uint32_t items_loaded = 0;
    WarpChunk wc_acc, wc_band;
    warp_chunk_init(wc_acc);
    warp_chunk_init(wc_band);

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            S.item = *abort ? 0xFFFFFFFFu : atomicAdd(a.head, 1u);
            S.max_e = S.max_n = S.max_r = 0u;
        }
        __syncthreads();
        const uint32_t item = S.item;
        if (item >= a.nblocks) break;
        const HjBlock blk = a.blocks[item];
        const uint32_t nq = blk.q1 - blk.q0;
        // query ids and block maxima of the error terms
        {
            float me = 0.f, mn = 0.f, mr = 0.f;
            for (uint32_t i = tid; i < (uint32_t)kQB; i += blockDim.x) {
                S.qid[i] = i < nq ? a.perm[blk.q0 + i] : 0u;
                if (i < nq) {
                    float4 p = a.pinfo[blk.q0 + i];
                    me = fmaxf(me, p.x); mn = fmaxf(mn, p.y); mr = fmaxf(mr, p.z);
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                me = fmaxf(me, __shfl_xor_sync(0xffffffffu, me, o));
                mn = fmaxf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            }
            if (lane == 0) {
                atomicMax(&S.max_e, __float_as_uint(me));
                atomicMax(&S.max_n, __float_as_uint(mn));
                atomicMax(&S.max_r, __float_as_uint(mr));
            }
        }
        if (warp == 0) {
            // stencil rows of the block's cell -> candidate ranges -> 128-row tiles
            const unsigned long long L = a.cell_lid[blk.cell];
            const uint32_t k = a.grid.k;
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
            if (empty) rows = 0;
            const StencilRows sr = stencil_rows(a.grid, lo, rows);
            uint32_t tiles_mine[kMaxRanges / 32];
            uint32_t my_tiles = 0;
#pragma unroll
            for (uint32_t s = 0; s < kMaxRanges / 32; ++s) {
                uint32_t r = lane * (kMaxRanges / 32) + s;
                uint32_t len = 0, st = 0;
                if (r < rows) {
                    const uint2 sp = cell_span(a.hash, a.cell_start, stencil_row_id(a.grid, sr, lo, w, r), w[0]);
                    st = sp.x;
                    len = sp.y - sp.x;
                    S.rs[r] = st;
                    S.rl[r] = len;
                }
                tiles_mine[s] = (len + kTileRows - 1) / kTileRows;
                my_tiles += tiles_mine[s];
            }
            uint32_t incl = my_tiles;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += t;
            }
            uint32_t run = incl - my_tiles;
            const uint32_t nr = min(rows, kMaxRanges);
#pragma unroll
            for (uint32_t s = 0; s < kMaxRanges / 32; ++s) {
                uint32_t r = lane * (kMaxRanges / 32) + s;
                if (r < nr) S.tp[r] = run;
                run += tiles_mine[s];
            }
            if (lane == 31) {
                S.tp[nr] = incl;
                S.ntiles = incl;
                S.nr = nr;
                S.nq = nq;
                S.q0 = blk.q0;
            }
        }
        __syncthreads();
        const uint32_t ntiles = S.ntiles;
        if (ntiles == 0) continue;

        if (warp == 0) {
            if (lane == 0) {
                // ---------------- TMA producer
                // both query tiles: rows past the item's queries are masked in the epilogue,
                // rows past n are zero-filled
                tc::mbar_arrive_expect_tx(&S.bfull, kQT * tile_bytes);
                for (uint32_t j = 0; j < (uint32_t)kQT; ++j)
                    for (uint32_t kb = 0; kb < a.nkb; ++kb)
                        tc::tma_load_2d(b_tiles + kb * kBKBlockBytes + j * kKBlockBytes, &tm_query, &S.bfull,
                                        (int)(kb * 32), (int)(blk.q0 + j * kTileRows));
                TileWalk tw;
                for (uint32_t t = 0; t < ntiles; ++t) {
                    const uint32_t s = it % a.stages, use = it / a.stages;
                    if (use > 0 && !tc::mbar_wait(&S.empty_a[s], (use - 1) & 1u, abort, a.err, a.wait_cycles)) break;
                    tw.locate(S, t);
                    tc::mbar_arrive_expect_tx(&S.full_a[s], tile_bytes);
                    for (uint32_t kb = 0; kb < a.nkb; ++kb)
                        tc::tma_load_2d(a_tiles + s * tile_bytes + kb * kKBlockBytes, &tm_cand, &S.full_a[s],
                                        (int)(kb * 32), (int)tw.start);
                    ++it;
                }
            }
            __syncwarp();
            it = __shfl_sync(0xffffffffu, it, 0);
        } else if (warp <= kAcc) {
            if (lane == 0) {
                // ---------------- MMA issuer h (warp 1: h = 0, warp 2: h = 1) of the tiles t with
                // t % 2 == h, into accumulator h.  Two issuers: every barrier wait stalls the
                // issuing thread's MMA stream for ~160 cycles (measured), and the other issuer
                // keeps the tensor pipe busy meanwhile.
                const uint32_t h = warp - 1;
                bool ok = tc::mbar_wait(&S.bfull, items_loaded & 1u, abort, a.err, a.wait_cycles);
                tc::fence_after();
                const uint32_t ksteps = a.nkb * 2;
                const uint32_t a_base = tc::smem_u32(a_tiles), b_base = tc::smem_u32(b_tiles);
                for (uint32_t t = 0; ok && t < ntiles; ++t) {
                    const uint32_t s = it % a.stages, use = it / a.stages;
                    ++it;
                    if ((t & 1u) != h) continue;
                    if (!tc::mbar_wait(&S.full_a[s], use & 1u, abort, a.err, a.wait_cycles)) break;
                    if (acc_use[h] > 0 &&
                        !tc::mbar_wait(&S.empty_acc[h], (acc_use[h] - 1) & 1u, abort, a.err, a.wait_cycles))
                        break;
                    tc::fence_after();
                    // M = 128 candidates x N = 256 queries per MMA: the shape that keeps the
                    // tensor pipe busy (N = 128 MMAs issue at well under half its rate)
                    for (uint32_t ks = 0; ks < ksteps; ++ks) {
                        const uint32_t kin = (ks & 1u) * 32u;
                        uint64_t ad = tc::desc_kmajor_sw64(a_base + s * tile_bytes + (ks >> 1) * kKBlockBytes + kin);
                        uint64_t bd = tc::desc_kmajor_sw64(b_base + (ks >> 1) * kBKBlockBytes + kin);
                        tc::mma_f16(tmem + h * kAccCols, ad, bd, a.idesc, ks > 0 ? 1u : 0u);
                    }
                    tc::mma_commit(&S.full_acc[h]);
                    ++acc_use[h];
                    tc::mma_commit(&S.empty_a[s]);
                }
            }
            __syncwarp();
            it = __shfl_sync(0xffffffffu, it, 0);
#pragma unroll
            for (int j = 0; j < kAcc; ++j) acc_use[j] = __shfl_sync(0xffffffffu, acc_use[j], 0);
            ++items_loaded;
        } else {
            // ---------------- epilogue: warps 3 .. 3 + 4*EPI.  SPLIT: two sets of 2*EPI warps,
            // one per accumulator (tiles of one parity), so a warp has two tiles' MMA time to
            // drain its share and a slow warp holds back only its own accumulator; otherwise
            // one set of 4*EPI warps drains every tile.  TMEM lane quarter = warp % 4; column
            // group within the set = (index in set) / 4.
            constexpr uint32_t SETW = SPLIT ? 2 * EPI : 4 * EPI;
            const uint32_t ew = warp - 1 - kAcc;
            const uint32_t hset = ew / SETW;   // SPLIT: the accumulator (tile parity) this warp drains
            const uint32_t quarter = warp & 3u;
            const uint32_t grp = (ew % SETW) >> 2;
            const uint32_t row = quarter * 32u + lane;
            const uint32_t lane_base = (quarter * 32u) << 16;
            // per-thread pair counts of one launch stay far below 2^32 (bounded by the sink)
            uint32_t n_acc = 0, n_band = 0;
            bool ok = true;
            // this warp's columns of an accumulator: COLS = 256 / (SETW / 4), read in chunks
            // of LDW by tcgen05.ld, W chunks per wait ("wave").
            constexpr uint32_t COLS = kAccCols / (SETW / 4);
            constexpr uint32_t LDW = EPI == 4 ? 32u : 64u;
            constexpr uint32_t NCH = COLS / LDW;
            constexpr uint32_t W = (EPI == 2 || !SPLIT) ? 2u : 1u;
            static_assert(NCH % W == 0, "whole waves per accumulator");
            const uint32_t t_first = SPLIT ? hset : 0u, t_step = SPLIT ? 2u : 1u;
            const uint32_t ncols = min((uint32_t)kAccCols, S.nq);
            const uint32_t q0 = S.q0;
            // the query block's part of the guard band, added to the threshold once per item
            const float qb = __double2float_ru(tc_band_q(a.gamma_acc, a.s_t, a.ref_rel, __uint_as_float(S.max_e),
                                                         __uint_as_float(S.max_n), __uint_as_float(S.max_r)));
            const float thr_hi = __fadd_ru(a.thr, qb), thr_lo = __fsub_rd(a.thr, qb);
            TileWalk tw;
            // the row's band term and original id, loaded one tile ahead: a global load on
            // the hit path stalls the warp, and a stalled warp holds back the release of the
            // next accumulator
            float pb_next = 0.f;
            uint32_t cid_next = 0u;
            if (t_first < ntiles) {
                tw.locate(S, t_first);
                if (row < tw.valid) {
                    pb_next = a.pband[tw.start + row];
                    if (!a.count_only) cid_next = a.perm[tw.start + row];
                }
            }
            for (uint32_t t = t_first; ok && t < ntiles; t += t_step) {
                const uint32_t j = t & 1u;
                const uint32_t cpos = tw.start + row;
                const bool vrow = row < tw.valid;
                const float hi = vrow ? __fadd_ru(thr_hi, pb_next) : -INFINITY;
                const float lo = vrow ? __fsub_rd(thr_lo, pb_next) : -INFINITY;
                const uint32_t cid = cid_next;   // the owner lane's id reaches the writing lane by a shuffle
                if (t + t_step < ntiles) {
                    // the next tile's rows, loaded while this tile is processed
                    tw.locate(S, t + t_step);
                    if (row < tw.valid) {
                        pb_next = a.pband[tw.start + row];
                        if (!a.count_only) cid_next = a.perm[tw.start + row];
                    }
                }
                if (!tc::mbar_wait(&S.full_acc[j], acc_use[j] & 1u, abort, a.err, a.wait_cycles)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                if constexpr (DEFER) {
                    // fast pass: min-reduce every chunk and note, per row, the chunks with a value
                    // not above the upper band edge; no vote or branch per chunk
                    uint32_t hitw = 0;
                    auto load_chunk = [&](float (&v)[LDW], uint32_t c) {
                        const uint32_t col = grp * COLS + c * LDW;
                        if constexpr (LDW == 64) tc::tmem_ld_32x64(tmem + lane_base + j * kAccCols + col, v);
                        else tc::tmem_ld_32x32(tmem + lane_base + j * kAccCols + col, v);
                    };
#pragma unroll
                    for (uint32_t c0 = 0; c0 < NCH; c0 += W) {
                        float v[W][LDW];
#pragma unroll
                        for (uint32_t w = 0; w < W; ++w) load_chunk(v[w], c0 + w);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (uint32_t w = 0; w < W; ++w) hitw |= (uint32_t)not_above(minN<LDW>(v[w]), hi) << (c0 + w);
                    }
                    // chunks where some row hit are read again (rare: the accumulator is still
                    // held) and classified pair by pair
                    uint32_t wave_hits = __reduce_or_sync(0xffffffffu, hitw);
                    while (wave_hits) {
                        const uint32_t c = __ffs(wave_hits) - 1;
                        wave_hits &= wave_hits - 1;
                        float v[LDW];
                        load_chunk(v, c);
                        tc::tmem_ld_wait();
                        const bool any_hit = (hitw >> c) & 1u;
                        const uint32_t col0 = grp * COLS + c * LDW;
#pragma unroll
                        for (uint32_t h = 0; h < LDW / 32; ++h) {
                            const uint32_t qcol = col0 + h * 32u;
                            uint32_t hmask = 0, amask = 0;
                            if (any_hit) {
#pragma unroll
                                for (int i = 0; i < 32; ++i) {
                                    bool inq = qcol + i < ncols;
                                    hmask |= (uint32_t)(inq && not_above(v[h * 32 + i], hi)) << i;
                                    amask |= (uint32_t)(inq && v[h * 32 + i] <= lo) << i;
                                }
                            }
                            const uint32_t bmask = hmask & ~amask;
                            n_acc += __popc(amask);
                            n_band += __popc(bmask);
                            if (a.count_only) continue;
                            // coalesced output: each lane writes every 32nd pair of the warp's
                            // hits; the owner lane's row gives the candidate
                            warp_emit_masks_v(a.sink, wc_acc, amask, cid, [&](uint32_t, uint32_t b, uint32_t ocid) {
                                return make_uint2(S.qid[qcol + b], ocid);
                            });
                            warp_emit_masks_v(a.band, wc_band, bmask, cpos, [&](uint32_t, uint32_t b, uint32_t opos) {
                                return make_uint2(q0 + qcol + b, opos);
                            });
                        }
                    }
                    // every column of this warp has been read: release the accumulator
                    tc::fence_before();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&S.empty_acc[j]);
                } else {
                    // per chunk: min-reduce, vote, and classify at once; the accumulator is
                    // released as soon as the last wave is in registers
#pragma unroll 1
                    for (uint32_t c0 = 0; c0 < NCH; c0 += W) {
                        float v[W][LDW];
#pragma unroll
                        for (uint32_t w = 0; w < W; ++w) {
                            const uint32_t col = grp * COLS + (c0 + w) * LDW;
                            if constexpr (LDW == 64) {
                                tc::tmem_ld_32x64(tmem + lane_base + j * kAccCols + col, v[w]);
                            } else {
                                tc::tmem_ld_32x32(tmem + lane_base + j * kAccCols + col, v[w]);
                            }
                        }
                        tc::tmem_ld_wait();
                        if (c0 + W >= NCH) {
                            // all of this warp's columns are in registers: release the accumulator
                            tc::fence_before();
                            __syncwarp();
                            if (lane == 0) tc::mbar_arrive(&S.empty_acc[j]);
                        }
#pragma unroll
                        for (uint32_t w = 0; w < W; ++w) {
                            const uint32_t col0 = grp * COLS + (c0 + w) * LDW;
                            const bool any_hit = not_above(minN<LDW>(v[w]), hi);
                            if (!__any_sync(0xffffffffu, any_hit)) continue;
#pragma unroll
                            for (uint32_t h = 0; h < LDW / 32; ++h) {
                                const uint32_t qcol = col0 + h * 32u;
                                uint32_t hmask = 0, amask = 0;
                                if (any_hit) {
#pragma unroll
                                    for (int i = 0; i < 32; ++i) {
                                        bool inq = qcol + i < ncols;
                                        hmask |= (uint32_t)(inq && not_above(v[w][h * 32 + i], hi)) << i;
                                        amask |= (uint32_t)(inq && v[w][h * 32 + i] <= lo) << i;
                                    }
                                }
                                const uint32_t bmask = hmask & ~amask;
                                n_acc += __popc(amask);
                                n_band += __popc(bmask);
                                if (a.count_only) continue;
                                // coalesced output: each lane writes every 32nd pair of the warp's
                                // hits; the owner lane's row gives the candidate
                                warp_emit_masks_v(a.sink, wc_acc, amask, cid, [&](uint32_t, uint32_t b, uint32_t ocid) {
                                    return make_uint2(S.qid[qcol + b], ocid);
                                });
                                warp_emit_masks_v(a.band, wc_band, bmask, cpos, [&](uint32_t, uint32_t b, uint32_t opos) {
                                    return make_uint2(q0 + qcol + b, opos);
                                });
                            }
                        }
                    }
                }
                ++acc_use[j];
            }
            unsigned long long w_acc = n_acc, w_band = n_band;
            for (int o = 16; o > 0; o >>= 1) {
                w_acc += __shfl_down_sync(0xffffffffu, w_acc, o);
                w_band += __shfl_down_sync(0xffffffffu, w_band, o);
            }
            if (lane == 0) {
                if (a.count_only) {
                    if (w_acc + w_band) atomicAdd(&a.block_counts[item], w_acc + w_band);
                } else if (a.stats) {
                    if (w_acc) atomicAdd(&a.stats[0], w_acc);
                    if (w_band) atomicAdd(&a.stats[1], w_band);
                }
            }
            it += ntiles;
        }
    }
    if (warp > kAcc && !a.count_only) {
        warp_chunk_close(a.sink, wc_acc);
        warp_chunk_close(a.band, wc_band);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

// Band pairs: exact FP32 refine in the reference's order (kernel.cu:350-355).
__global__ void k_band_recheck(const float* __restrict__ pts, const uint32_t* __restrict__ perm, uint32_t d,
                               float thr, const uint32_t* __restrict__ bq, const uint32_t* __restrict__ bc,
                               const unsigned long long* __restrict__ band_used, unsigned long long band_cap,
                               PairSink sink) {
    const unsigned long long n = min(*band_used, band_cap);
    WarpChunk wc;
    warp_chunk_init(wc);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < n; base += stride) {
        unsigned long long i = base + threadIdx.x;
        bool hit = false;
        uint32_t qp = 0, cp = 0;
        if (i < n) {
            qp = bq[i];
            if (qp != kSentinelKey) {
                cp = bc[i];
                const float* q = pts + (size_t)qp * d;
                const float* c = pts + (size_t)cp * d;
                float acc = 0.f;
                for (uint32_t l = 0; l < d; ++l) {
                    float diff = __fsub_rn(c[l], q[l]);
                    acc = __fmaf_rn(diff, diff, acc);
                }
                hit = acc <= thr;
            }
        }
        warp_emit(sink, wc, hit ? 1u : 0u, [&](uint32_t) { return make_uint2(perm[qp], perm[cp]); });
    }
    warp_chunk_close(sink, wc);
}

// Operand preparation: one thread per sorted point.
template <typename H>
__device__ __forceinline__ H to_h(double x);
template <>
__device__ __forceinline__ __half to_h<__half>(double x) { return __double2half(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 to_h<__nv_bfloat16>(double x) { return __double2bfloat16(x); }
__device__ __forceinline__ double from_h(__half h) { return (double)__half2float(h); }
__device__ __forceinline__ double from_h(__nv_bfloat16 h) { return (double)__bfloat162float(h); }

// Block-wide maximum of non-negative values, folded into *out with one atomic
// per block (non-negative IEEE values order like their bit patterns).
__device__ __forceinline__ void block_max_into(double v, unsigned long long* out) {
    __shared__ double part[32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane_id() == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v > 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

// Largest |x - origin|^2 over the points, in FP64 (the scale of the operand
// forms is chosen from it), and whether any coordinate is not finite.
__global__ void k_tc_range(const float* __restrict__ pts, uint32_t n, uint32_t d, const float* __restrict__ origin,
                           unsigned long long* __restrict__ max_n2, uint32_t* __restrict__ nonfinite) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double n2 = 0;
    bool bad = false;
    if (i < n) {
        for (uint32_t l = 0; l < d; ++l) {
            const float v = pts[i * d + l];
            bad |= !isfinite(v);
            const double x = (double)v - (double)origin[l];
            n2 += x * x;
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane_id() == 0) atomicOr(nonfinite, 1u);
    block_max_into(bad ? 0.0 : n2, max_n2);
}

// Operand forms of one sorted point (one thread each), in units scaled by
// `scale` (a power of two): x~ = half((x - origin) * scale).  Also folds the
// maxima of the per-point bound terms into maxima[0..2] (float bits).
template <typename H>
__global__ void k_tc_prep(const float* __restrict__ pts, uint32_t n, uint32_t d, uint32_t kpad,
                          const float* __restrict__ origin, double scale, H* __restrict__ qform,
                          H* __restrict__ cform, float4* __restrict__ pinfo, unsigned int* __restrict__ maxima) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i < n) {
        double n2 = 0, e2 = 0;
        H* qr = qform + (size_t)i * kpad;
        H* cr = cform + (size_t)i * kpad;
        for (uint32_t l = 0; l < d; ++l) {
            double x = ((double)pts[(size_t)i * d + l] - (double)origin[l]) * scale;   // exact: scale is 2^s
            H h = to_h<H>(x);
            double xt = from_h(h);
            e2 += (xt - x) * (xt - x);
            n2 += xt * xt;
            qr[l] = h;
            cr[l] = to_h<H>(-2.0 * xt);
        }
        H nh = to_h<H>(n2);
        H nl = to_h<H>(n2 - from_h(nh));
        double res = fabs(n2 - from_h(nh) - from_h(nl));
        H one = to_h<H>(1.0), zero = to_h<H>(0.0);
        qr[d] = nh; qr[d + 1] = nl; qr[d + 2] = one; qr[d + 3] = one;
        cr[d] = one; cr[d + 1] = one; cr[d + 2] = nh; cr[d + 3] = nl;
        for (uint32_t l = d + 4; l < kpad; ++l) { qr[l] = zero; cr[l] = zero; }
        // round the bounds up: float conversion is to nearest, so scale by 1 + 2^-20
        const float up = 1.0f + 9.6e-7f;
        p = make_float4((float)sqrt(e2) * up, (float)n2 * up, (float)res * up + 1e-30f, 0.f);
        pinfo[i] = p;
    }
    float m[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        float v = m[j];
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane_id() == 0 && v > 0.f) atomicMax(&maxima[j], __float_as_uint(v));
    }
}

// Each point's part of the guard band (tc_band_p), rounded up.
__global__ void k_tc_pband(const float4* __restrict__ pinfo, uint32_t n, double gamma, double s_t, double ref_rel,
                           float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pinfo[i];
    out[i] = __double2float_ru(tc_band_p(gamma, s_t, ref_rel, p.x, p.y, p.z));
}

// Per-dimension minimum of the points: lanes walk a row's dimensions (coalesced
// reads), warps stride over rows, one atomic per (block, dimension).
__global__ void k_col_min(const float* __restrict__ pts, uint32_t n, uint32_t d, float* __restrict__ out) {
    extern __shared__ float part[];   // [warps][d]
    const uint32_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
    for (uint32_t l = lane_id(); l < d; l += 32) part[w * d + l] = INFINITY;
    for (uint32_t i = blockIdx.x * warps + w; i < n; i += gridDim.x * warps)
        for (uint32_t l = lane_id(); l < d; l += 32) part[w * d + l] = fminf(part[w * d + l], pts[(size_t)i * d + l]);
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < d; l += blockDim.x) {
        float m = INFINITY;
        for (uint32_t k = 0; k < warps; ++k) m = fminf(m, part[k * d + l]);
        // non-negative floats order like their bit patterns as ints; negative ones
        // order in reverse as unsigned ints
        if (m >= 0.f) atomicMin(reinterpret_cast<int*>(out) + l, __float_as_int(m));
        else atomicMax(reinterpret_cast<unsigned int*>(out) + l, __float_as_uint(m));
    }
}

__global__ void k_fill_f32(float* p, uint32_t n, float v) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Debug/test kernel: one candidate tile (rows a0..a0+127) against four query
// tiles (rows b0..b0+511) through the same TMA maps, descriptors and MMA
// sequence as k_refine_tc; writes every accumulator value to out[128][512].
__global__ void __launch_bounds__(kProbeThreads, 1)
    k_tc_tile_probe(const __grid_constant__ CUtensorMap tm_cand, const __grid_constant__ CUtensorMap tm_query,
                    uint32_t nkb, uint32_t idesc, uint32_t a0, uint32_t b0, float* __restrict__ out, uint32_t* err,
                    uint32_t skip_mma, long long wait_cycles) {
    extern __shared__ uint8_t smem_raw[];
    uint32_t base = tc::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (base & 1023u)) & 1023u);
    const uint32_t tile_bytes = nkb * kKBlockBytes;
    uint8_t* b_tiles = smem;
    uint8_t* a_tile = smem + kProbeQT * tile_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(a_tile + tile_bytes);   // [0] loads, [1] mma
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    uint32_t* abortp = tslot + 1;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        *abortp = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(tslot, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    if (tid == 0) {
        tc::mbar_arrive_expect_tx(&bars[0], (kProbeQT + 1) * tile_bytes);
        for (uint32_t kb = 0; kb < nkb; ++kb) {
            tc::tma_load_2d(a_tile + kb * kKBlockBytes, &tm_cand, &bars[0], (int)(kb * 32), (int)a0);
            for (uint32_t j = 0; j < kProbeQT; ++j)
                tc::tma_load_2d(b_tiles + kb * kProbeBKBlockBytes + j * kKBlockBytes, &tm_query, &bars[0], (int)(kb * 32),
                                (int)(b0 + j * kTileRows));
        }
    }
    if (tid == 32) {
        // the loads always complete before this thread goes on, so with skip_mma no
        // TMA transfer is in flight while the epilogue's wait runs out
        bool ok = tc::mbar_wait(&bars[0], 0, abortp, err, wait_cycles);
        tc::fence_after();
        if (ok && !skip_mma) {
            for (uint32_t j = 0; j < kAcc; ++j)
                for (uint32_t ks = 0; ks < nkb * 2; ++ks) {
                    const uint32_t kin = (ks & 1u) * 32u;
                    tc::mma_f16(tmem + j * kAccCols,
                                tc::desc_kmajor_sw64(tc::smem_u32(a_tile) + (ks >> 1) * kKBlockBytes + kin),
                                tc::desc_kmajor_sw64(tc::smem_u32(b_tiles) + (ks >> 1) * kProbeBKBlockBytes +
                                                     j * (kAccCols * 64u) + kin),
                                idesc, ks > 0 ? 1u : 0u);
                }
        }
        // skip_mma: no MMA and no commit, so the wait below runs out (the timeout test)
        if (!skip_mma) tc::mma_commit(&bars[1]);
    }
    if (warp >= 2) {
        const uint32_t quarter = warp & 3u;
        bool ok = tc::mbar_wait(&bars[1], 0, abortp, err, wait_cycles);
        tc::fence_after();
        if (ok) {
            for (uint32_t col = 0; col < (uint32_t)kProbeQB; col += 32) {
                float v[32];
                tc::tmem_ld_32x32(tmem + ((quarter * 32u) << 16) + col, v);
                tc::tmem_ld_wait();
#pragma unroll
                for (int i = 0; i < 32; ++i) out[(size_t)(quarter * 32 + lane) * kProbeQB + col + i] = v[i];
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

// ---- host side -------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

hj_status make_map(CUtensorMap* m, const void* base, uint32_t rows, uint32_t kpad, int kind) {
    auto fn = encode_fn();
    if (!fn) { set_error("cuTensorMapEncodeTiled is not available"); return HJ_ERR_CUDA; }
    cuuint64_t dims[2] = {kpad, rows};
    cuuint64_t strides[1] = {(cuuint64_t)kpad * 2};
    cuuint32_t box[2] = {32, (cuuint32_t)kTileRows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, kind == HJ_REFINE_TC_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                    2, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return HJ_ERR_CUDA;
    }
    return HJ_OK;
}

uint32_t kpad_for(uint32_t d) { return ((d + 4 + 31) / 32) * 32; }

// The float constants of the guard band, shared by the per-point terms and the kernel.
float band_s_t(double thr_s) { return (float)(std::sqrt(thr_s * (1 + 1e-4)) * (1 + 1e-6)); }   // sqrt(T (1 + 1e-4))
float band_ref_rel(uint32_t d) { return (float)((d + 2) * std::ldexp(1.0, -24) * 1.01); }
// Accumulation model: each K=16 MMA step adds 16 exact products to the FP32
// accumulator with at most 2 ulps of the largest magnitude per term lost
// (alignment and truncation); bound = (steps + 1) * 32 * 2^-23 * sum|terms|.
float band_gamma(uint32_t kpad) { return (float)((kpad / 16 + 1) * 32 * std::ldexp(1.0, -23)); }

size_t tc_smem_bytes(uint32_t nkb, uint32_t stages) {
    return 1024 + (size_t)(kQT + stages) * nkb * kKBlockBytes + sizeof(TcShared);
}

uint32_t tc_stages(uint32_t nkb) {
    size_t budget = 225 * 1024;
    uint32_t s = kMaxStages;
    while (s > 2 && tc_smem_bytes(nkb, s) > budget) --s;
    return s;
}

struct TcMaps {
    CUtensorMap cand, query;
};

}  // namespace

struct TcState {
    TcMaps maps;
    int epi = 4;              // epilogue shape code, EPI | 8 * SPLIT (autotuned: 2, 4, 10, 12)
    bool defer = false;       // one vote per accumulator (set from the estimated pair density)
    float gamma_acc = 0;
    int scale_exp = 0;        // operand forms hold (x - origin) * 2^scale_exp
    double thr_s = 0;         // the squared threshold in those units: thr * 4^scale_exp, exact
    float max_e = 0, max_n = 0, max_r = 0;   // maxima of the per-point bound terms (scaled units)
};

static TcState* tc_state(const hj_index* ix) { return reinterpret_cast<TcState*>(ix->tc_state); }

bool tc_supported(const hj_index* ix, int kind) {
    if (ix->dtype != HJ_F32 || ix->d < 8) return false;
    if (kind != HJ_REFINE_TC_F16 && kind != HJ_REFINE_TC_BF16) return false;
    uint32_t nkb = kpad_for(ix->d) / 32;
    if (tc_smem_bytes(nkb, 2) > 225 * 1024) return false;
    uint32_t rows = 1;
    for (uint32_t j = 1; j < ix->k; ++j) rows *= 3;
    return rows <= kMaxRanges && ix->n < 0x7FFFFF00u;
}

uint32_t tc_query_block() { return kQB; }

// Band recheck grid for a refine over nblocks work items: as many blocks as there
// are SMs x 8, but no more than 8 per refine CTA (small joins have small bands).
static unsigned recheck_grid(uint32_t nblocks) {
    return (unsigned)std::min<uint64_t>((uint64_t)num_sms() * 8, 8ull * std::max<uint32_t>(1, std::min<uint32_t>(nblocks, num_sms())));
}

// Upper bound on the warps that reserve chunks of one sink during one batch: the
// refine's epilogue warps (at most 16 per CTA, one CTA per SM) and the band
// recheck's warps (8 per block), each holding at most one partly filled chunk.
uint64_t tc_emit_warps(uint32_t nblocks) {
    return (uint64_t)std::min<uint32_t>((uint32_t)num_sms(), std::max<uint32_t>(nblocks, 1)) * 16ull +
           (uint64_t)recheck_grid(nblocks) * 8ull;
}

// Half-width of the guard band for the worst pair of the dataset, in scaled units.
static double tc_delta_scaled(const hj_index* ix, const TcState* s) {
    const double sT = band_s_t(s->thr_s), ref = band_ref_rel(ix->d), g = s->gamma_acc;
    return tc_band_p(g, sT, ref, s->max_e, s->max_n, s->max_r) + tc_band_q(g, sT, ref, s->max_e, s->max_n, s->max_r);
}

// The same in the dataset's units (the figure the join reports).
double tc_delta(const hj_index* ix) {
    TcState* s = tc_state(ix);
    if (!s) return 0;
    return std::ldexp(tc_delta_scaled(ix, s), -2 * s->scale_exp);
}

// Band half-width over the threshold: where it is large the filter decides
// little and nearly every neighbour goes through the exact recheck.
double tc_band_ratio(const hj_index* ix) {
    TcState* s = tc_state(ix);
    if (!s) return 1e300;
    return s->thr_s > 0 ? tc_delta_scaled(ix, s) / s->thr_s : 1e300;
}

int tc_scale_exp(const hj_index* ix) {
    TcState* s = tc_state(ix);
    return s ? s->scale_exp : 0;
}

void tc_release(hj_index* ix) {
    delete tc_state(ix);
    ix->tc_state = nullptr;
}

// Power-of-two exponent s for the operand forms: the largest |x - origin|^2
// times 4^s lands in (2^12, 2^14], and the threshold times 4^s stays a normal
// float (so scaling it is exact).  Returns false when both cannot hold.
static bool choose_scale(double max_n2, double thr, int* out) {
    int s = 0;
    if (max_n2 > 0) {
        int e2 = 0;
        std::frexp(max_n2, &e2);                 // max_n2 in [2^(e2-1), 2^e2)
        s = (14 - e2) >> 1;                      // floor((14 - e2) / 2)
        while (s > -600 && std::ldexp(max_n2, 2 * s) > 16384.0) --s;
        while (s < 600 && std::ldexp(max_n2, 2 * s + 2) <= 16384.0) ++s;
    }
    if (thr > 0) {
        // keep T * 4^s within [2^-100, 2^100]: exact in float and far from overflow
        while (std::ldexp(thr, 2 * s) > std::ldexp(1.0, 100)) --s;
        if (std::ldexp(thr, 2 * s) < std::ldexp(1.0, -100)) return false;
    }
    if (max_n2 > 0 && std::ldexp(max_n2, 2 * s) > 16384.0 * 1.0001) return false;
    *out = s;
    return true;
}

hj_status tc_prepare(hj_index* ix, int kind, cudaStream_t st) {
    if (ix->tc_kind == kind && ix->tc_state) return HJ_OK;
    // Drop the previous operand forms before anything else: if a step below
    // fails, no tensor map may be left pointing at freed buffers.
    tc_release(ix);
    ix->tc_kind = -1;
    dfree(ix->tc_a, st);
    dfree(ix->tc_b, st);
    dfree(ix->tc_err, st);
    dfree(ix->tc_pband, st);
    const uint32_t kpad = kpad_for(ix->d), n = ix->n, d = ix->d;
    uint16_t *qf = nullptr, *cf = nullptr;
    float* origin = nullptr;
    float4* pinfo = nullptr;
    float* pband = nullptr;
    unsigned long long* rng = nullptr;   // [0] max |x - origin|^2 (FP64 bits), [1] non-finite flag
    unsigned int* mx = nullptr;          // maxima of the bound terms (float bits)
    auto fail = [&](hj_status e) {
        cudaGetLastError();
        dfree(qf, st); dfree(cf, st); dfree(pinfo, st); dfree(origin, st); dfree(rng, st); dfree(mx, st);
        dfree(pband, st);
        return e;
    };
#define TC_TRY(x) do { hj_status e_ = (x); if (e_ != HJ_OK) return fail(e_); } while (0)
    TC_TRY(dalloc(&qf, (size_t)n * kpad, st));
    TC_TRY(dalloc(&cf, (size_t)n * kpad, st));
    TC_TRY(dalloc(&pinfo, n, st));
    TC_TRY(dalloc(&pband, n, st));
    TC_TRY(dalloc(&origin, d, st));
    TC_TRY(dalloc(&rng, 2, st));
    TC_TRY(dalloc(&mx, 4, st));
    TC_TRY(cuda_status(cudaMemsetAsync(rng, 0, 2 * sizeof(unsigned long long), st), "clear range scratch"));
    TC_TRY(cuda_status(cudaMemsetAsync(mx, 0, 4 * sizeof(unsigned int), st), "clear maxima"));
    k_fill_f32<<<(d + 255) / 256, 256, 0, st>>>(origin, d, INFINITY);
    TC_TRY(launch_status(__FILE__, __LINE__));
    {
        const unsigned blocks = (unsigned)std::min<uint32_t>(num_sms() * 2, std::max<uint32_t>(1, n / 64));
        k_col_min<<<blocks, 256, (size_t)8 * d * sizeof(float), st>>>((const float*)ix->pts, n, d, origin);
        TC_TRY(launch_status(__FILE__, __LINE__));
    }
    const unsigned pblocks = std::max<uint32_t>(1, (n + 255) / 256);
    k_tc_range<<<pblocks, 256, 0, st>>>((const float*)ix->pts, n, d, origin, rng,
                                        reinterpret_cast<uint32_t*>(rng + 1));
    TC_TRY(launch_status(__FILE__, __LINE__));
    unsigned long long hr[2] = {0, 0};
    TC_TRY(cuda_status(cudaMemcpyAsync(hr, rng, sizeof(hr), cudaMemcpyDeviceToHost, st), "range to host"));
    TC_TRY(cuda_status(cudaStreamSynchronize(st), "range sync"));
    if (hr[1]) {
        set_error("the tensor-core filter needs finite coordinates (the dataset holds inf or NaN)");
        return fail(HJ_ERR_UNSUPPORTED);
    }
    double max_n2 = 0;
    std::memcpy(&max_n2, &hr[0], sizeof(double));
    int sexp = 0;
    if (!choose_scale(max_n2, ix->thr, &sexp)) {
        set_error("the tensor-core filter cannot scale this dataset: eps^2 / max |x - min|^2 = %g is below 2^-114",
                  ix->thr / max_n2);
        return fail(HJ_ERR_UNSUPPORTED);
    }
    const double scale = std::ldexp(1.0, sexp);
    if (kind == HJ_REFINE_TC_BF16)
        k_tc_prep<__nv_bfloat16><<<pblocks, 256, 0, st>>>((const float*)ix->pts, n, d, kpad, origin, scale,
                                                           (__nv_bfloat16*)qf, (__nv_bfloat16*)cf, pinfo, mx);
    else
        k_tc_prep<__half><<<pblocks, 256, 0, st>>>((const float*)ix->pts, n, d, kpad, origin, scale, (__half*)qf,
                                                    (__half*)cf, pinfo, mx);
    TC_TRY(launch_status(__FILE__, __LINE__));
    unsigned int hm[4] = {0, 0, 0, 0};
    TC_TRY(cuda_status(cudaMemcpyAsync(hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, st), "maxima to host"));
    TC_TRY(cuda_status(cudaStreamSynchronize(st), "maxima sync"));
    TcMaps maps;
    TC_TRY(make_map(&maps.query, qf, n, kpad, kind));
    TC_TRY(make_map(&maps.cand, cf, n, kpad, kind));
    // each point's part of the guard band
    const float gamma_acc = band_gamma(kpad);
    const double thr_s = std::ldexp(ix->thr, 2 * sexp);
    k_tc_pband<<<pblocks, 256, 0, st>>>(pinfo, n, gamma_acc, band_s_t(thr_s), band_ref_rel(d), pband);
    TC_TRY(launch_status(__FILE__, __LINE__));
#undef TC_TRY
    dfree(origin, st);
    dfree(rng, st);
    dfree(mx, st);
    TcState* s = new TcState();
    s->maps = maps;
    s->gamma_acc = gamma_acc;
    s->scale_exp = sexp;
    s->thr_s = thr_s;
    std::memcpy(&s->max_e, &hm[0], 4);
    std::memcpy(&s->max_n, &hm[1], 4);
    std::memcpy(&s->max_r, &hm[2], 4);
    ix->tc_a = qf;
    ix->tc_b = cf;
    ix->tc_err = reinterpret_cast<float*>(pinfo);
    ix->tc_pband = pband;
    ix->tc_kpad = kpad;
    ix->tc_state = s;
    ix->tc_kind = kind;
    return HJ_OK;
}

int tc_get_epi(const hj_index* ix) {
    TcState* s = tc_state(ix);
    return s ? s->epi : 0;
}
void tc_set_epi(hj_index* ix, int epi) {
    TcState* s = tc_state(ix);
    if (s && (epi == 2 || epi == 4 || epi == 10 || epi == 12)) s->epi = epi;
}

void tc_set_defer(hj_index* ix, bool defer) {
    TcState* s = tc_state(ix);
    if (s) s->defer = defer;
}

hj_status launch_refine_tc(const hj_index* ix, const HjBlock* blocks, uint32_t nblocks, unsigned int* head,
                           const PairSink& sink, const PairSink& band, uint32_t count_only,
                           unsigned long long* block_counts, unsigned long long* stats, uint32_t* err,
                           cudaStream_t st) {
    if (nblocks == 0) return HJ_OK;
    TcState* s = tc_state(ix);
    if (!s) { set_error("tensor-core operands not prepared"); return HJ_ERR_INVALID; }
    const uint32_t nkb = ix->tc_kpad / 32, stages = tc_stages(nkb);
    size_t smem = tc_smem_bytes(nkb, stages);
    // one CTA per SM: ask for more than half of the SM's shared memory
    smem = std::max<size_t>(smem, 116 * 1024);
    const int code = s->epi;
    auto kern = s->defer ? (code == 2    ? k_refine_tc<2, false, true>
                            : code == 10 ? k_refine_tc<2, true, true>
                            : code == 12 ? k_refine_tc<4, true, true>
                                         : k_refine_tc<4, false, true>)
                         : (code == 2    ? k_refine_tc<2, false, false>
                            : code == 10 ? k_refine_tc<2, true, false>
                            : code == 12 ? k_refine_tc<4, true, false>
                                         : k_refine_tc<4, false, false>);
    const int epi = (code & 7) == 2 ? 2 : 4;
    HJ_TRY(ensure_smem(kern, smem));
    TcArgs a{};
    a.blocks = blocks; a.nblocks = nblocks; a.head = head;
    a.perm = ix->perm; a.cell_lid = ix->cell_lid; a.cell_start = ix->cell_start; a.nC = ix->nC; a.grid = ix->grid;
    a.hash = cell_hash(ix);
    a.pinfo = reinterpret_cast<const float4*>(ix->tc_err);
    a.pband = ix->tc_pband;
    a.n = ix->n; a.nkb = nkb; a.stages = stages;
    a.thr = (float)s->thr_s;   // exact: thr * 4^s
    a.gamma_acc = s->gamma_acc;
    a.s_t = band_s_t(s->thr_s);
    a.ref_rel = band_ref_rel(ix->d);
    a.sink = sink; a.band = band;
    a.count_only = count_only; a.block_counts = block_counts; a.stats = stats; a.err = err;
    a.idesc = tc::idesc_f16(ix->tc_kind == HJ_REFINE_TC_BF16 ? 1u : 0u, kTileRows, kAccCols);
    a.wait_cycles = kWaitCycles;
    unsigned grid = (unsigned)std::min<uint32_t>((uint32_t)num_sms(), nblocks);
    kern<<<grid, 32 * (1 + kAcc) + 128 * epi, smem, st>>>(s->maps.cand, s->maps.query, a);
    HJ_LAUNCHED();
    return HJ_OK;
}

hj_status launch_band_recheck(const hj_index* ix, const uint32_t* bq, const uint32_t* bc,
                              const unsigned long long* band_used, unsigned long long band_cap, const PairSink& sink,
                              uint32_t nblocks, cudaStream_t st) {
    const unsigned grid = recheck_grid(nblocks);
    k_band_recheck<<<grid, 256, 0, st>>>((const float*)ix->pts, ix->perm, ix->d, (float)ix->thr, bq, bc, band_used,
                                         band_cap, sink);
    HJ_LAUNCHED();
    return HJ_OK;
}

}  // namespace hj

namespace hj {
// One launch of the tile probe.  skip_mma = 1 issues the loads but no MMA and no
// commit, so the epilogue's bounded wait runs out after wait_cycles.
static hj_status run_tile_probe(hj_index* ix, int kind, uint32_t a0, uint32_t b0, float* d_out, uint32_t skip_mma,
                                long long wait_cycles, void* h_query_rows, void* h_cand_rows, cudaStream_t st) {
    if (!ix || !d_out || !tc_supported(ix, kind)) { set_error("tensor-core tile probe: unsupported"); return HJ_ERR_INVALID; }
    HJ_TRY(tc_prepare(ix, kind, st));
    TcState* s = tc_state(ix);
    const uint32_t nkb = ix->tc_kpad / 32;
    size_t smem = 1024 + (size_t)(kProbeQT + 1) * nkb * kKBlockBytes + 64;
    smem = std::max<size_t>(smem, 116 * 1024);
    HJ_TRY(ensure_smem(k_tc_tile_probe, smem));
    Scratch tmp(st);
    uint32_t* err = nullptr;
    HJ_TRY(tmp.alloc(&err, 1));
    HJ_CUDA(cudaMemsetAsync(err, 0, 4, st));
    k_tc_tile_probe<<<1, kProbeThreads, smem, st>>>(s->maps.cand, s->maps.query, nkb,
                                               tc::idesc_f16(kind == HJ_REFINE_TC_BF16 ? 1u : 0u, kTileRows, kAccCols),
                                               a0, b0, d_out, err, skip_mma, wait_cycles);
    HJ_LAUNCHED();
    uint32_t herr = 0;
    HJ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
    if (h_query_rows)
        HJ_CUDA(cudaMemcpyAsync(h_query_rows, (const uint16_t*)ix->tc_a + (size_t)b0 * ix->tc_kpad,
                                (size_t)std::min<uint32_t>(kProbeQB, ix->n - b0) * ix->tc_kpad * 2, cudaMemcpyDeviceToHost, st));
    if (h_cand_rows)
        HJ_CUDA(cudaMemcpyAsync(h_cand_rows, (const uint16_t*)ix->tc_b + (size_t)a0 * ix->tc_kpad,
                                (size_t)std::min<uint32_t>(kTileRows, ix->n - a0) * ix->tc_kpad * 2,
                                cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("tensor-core tile probe: a bounded wait expired"); return HJ_ERR_TIMEOUT; }
    return HJ_OK;
}
}  // namespace hj

extern "C" hj_status hj_probe_tc_tile(hj_index* ix, int kind, uint32_t a0, uint32_t b0, float* d_out,
                                      void* h_query_rows, void* h_cand_rows, void* stream) {
    using namespace hj;
    if (ix && (a0 >= ix->n || b0 >= ix->n)) { set_error("hj_probe_tc_tile: row out of range"); return HJ_ERR_INVALID; }
    return run_tile_probe(ix, kind, a0, b0, d_out, 0u, kWaitCycles, h_query_rows, h_cand_rows, as_stream(stream));
}

extern "C" hj_status hj_probe_tc_wait_timeout(hj_index* ix, int kind, uint64_t wait_cycles, void* stream) {
    using namespace hj;
    if (!ix || wait_cycles == 0 || wait_cycles > (uint64_t)kWaitCycles) {
        set_error("hj_probe_tc_wait_timeout: wait_cycles must be in [1, %lld]", kWaitCycles);
        return HJ_ERR_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    Scratch tmp(st);
    float* out = nullptr;
    HJ_TRY(tmp.alloc(&out, (size_t)kTileRows * kProbeQB));
    return run_tile_probe(ix, kind, 0, 0, out, 1u, (long long)wait_cycles, nullptr, nullptr, st);
}

extern "C" hj_status hj_tc_operand_scale(const hj_index* ix, int* log2_scale) {
    using namespace hj;
    if (!ix || !log2_scale) { set_error("hj_tc_operand_scale: null argument"); return HJ_ERR_INVALID; }
    if (!ix->tc_state) { set_error("hj_tc_operand_scale: no tensor-core operands prepared"); return HJ_ERR_INVALID; }
    *log2_scale = tc_scale_exp(ix);
    return HJ_OK;
}
