// hj_internal.h -- library-internal structures shared by the .cu files.
#pragma once

#include "hj_common.cuh"

// Grid parameters passed by value to kernels.
struct HjGrid {
    uint32_t k;
    uint32_t n_cells[hj::kMaxK];
    unsigned long long mult[hj::kMaxK];   // mixed-radix multipliers, dimension 0 fastest
    // Row offsets of a full stencil box (width 3 along every dimension j >= 1):
    // entry r is sum over j >= 1 of digit_j(r) * mult[j], the base-3 digits of r
    // with dimension 1 fastest; full_rows = 3^(k-1) entries.  Null (and
    // full_rows 0) for k > kRowOffMaxK.
    const unsigned long long* row_off;
    uint32_t full_rows;
};
constexpr uint32_t kRowOffMaxK = 7;   // at most 729 offsets

// Open-addressing hash of the non-empty cells, keyed by groups of four
// consecutive linear ids (g = lid >> 2).  An entry is 16 bytes: the group key
// (two words), the cell index of the group's first non-empty cell, and a 4-bit
// mask of the group's non-empty ids; the group's cells are consecutive in the
// cell table (sorted by linear id), so the cell of id g*4 + b is the first cell
// plus the number of mask bits below b.  A stencil row (up to 3 consecutive ids
// along dimension 0) spans one or two groups: one or two 16-byte loads, and
// neighbouring cells along dimension 0 hit the same entries.  Capacity is a
// power of two at least twice the number of cells (so at most half full of
// groups); free entries hold the key
// kEmptyLid (no group can have it: linear ids stay below 2^63).
// A table too large for L2 gets an occupancy filter beside it: two bits of one
// 32-bit word per group (16 bits per cell), set at insertion.  A probe of an
// absent group, the common case on sparse data, then costs one load of a
// filter small enough to stay in L2 instead of a random DRAM read of the table;
// about 2% of absent groups pass the filter and read the table as before.
struct HjCellHash {
    const uint4* entries;
    unsigned long long mask;       // capacity - 1
    const uint32_t* occ;           // occupancy filter, or null (small tables)
    unsigned long long occ_mask;   // filter words - 1
};

// Work item of the refine kernels: queries q0..q1 (sorted positions) of cell
// `cell`, whose stencil holds `nb` candidate points.
struct HjBlock {
    uint32_t cell;
    uint32_t q0;
    uint32_t q1;
    uint32_t nb;
};

struct hj_index {
    uint32_t n = 0, d = 0, k = 0;
    int dtype = HJ_F32;
    double eps = 0;            // value in dataset type
    double thr = 0;            // largest d2 with RN(sqrt(d2)) <= eps (dataset type)
    double min_arr[hj::kMaxK] = {};
    HjGrid grid = {};
    uint64_t total_cells = 0;
    uint32_t aliasing = 0;
    int device = 0;
    cudaStream_t stream = nullptr;   // stream the index was built on; its memory is freed in that order

    // device arrays
    void* pts = nullptr;             // n x d, dataset type, ordered by (cell id, original id)
    uint32_t* perm = nullptr;        // sorted position -> original id (indexLookupArr)
    unsigned long long* cell_lid = nullptr;  // nC sorted linear ids
    uint32_t* cell_start = nullptr;  // nC + 1
    uint32_t nC = 0;
    uint4* hash_entries = nullptr;   // cell hash (HjCellHash)
    unsigned long long hash_mask = 0;
    uint32_t* hash_occ = nullptr;    // its occupancy filter (large tables only)
    unsigned long long occ_mask = 0;
    unsigned long long* row_off = nullptr;   // grid.row_off

    // workload (hj_sort_by_workload)
    bool have_workload = false;
    uint64_t total_candidates = 0;
    uint32_t* cell_nb = nullptr;     // candidates per cell (cell order)
    uint32_t* cell_order = nullptr;  // cells, heaviest first
    uint32_t max_nb = 0;

    // tensor-core operands (built on first use)
    void* tc_a = nullptr;            // n x kpad, query form
    void* tc_b = nullptr;            // n x kpad, candidate form
    float* tc_err = nullptr;         // per sorted point: quantisation error norm (rounded up)
    float* tc_pband = nullptr;       // per sorted point: its part of the guard band (rounded up)
    uint32_t tc_kpad = 0;
    int plain_shape = 0;             // exact refine tile shape (0 or 1; autotuned per d and dtype)
    int tc_kind = -1;                // HJ_REFINE_TC_F16 / _BF16 the operands hold
    void* tc_state = nullptr;        // tensor maps and error maxima (hj_refine_tc.cu)
};

namespace hj {

// Host: largest value x of the dataset type with RN(sqrt(x)) <= eps.
double sq_threshold(double eps, int dtype);

// Keep freed stream-ordered allocations mapped for reuse (called once per process).
void init_memory_pool();

// hj_refine_tc.cu
void tc_release(hj_index* ix);

// hj_index.cu
hj_status build_blocks(const hj_index* ix, uint32_t qb, HjBlock** d_blocks, uint32_t* n_blocks,
                       cudaStream_t st);

constexpr unsigned long long kEmptyLid = ~0ull;
constexpr uint32_t kNoCell = 0xFFFFFFFFu;

inline HjCellHash cell_hash(const hj_index* ix) {
    return HjCellHash{ix->hash_entries, ix->hash_mask, ix->hash_occ, ix->occ_mask};
}

// The filter word of group g and the two bits the group sets in it (a second
// hash of g, independent of the slot index).
__host__ __device__ __forceinline__ void occ_bits(unsigned long long g, unsigned long long occ_mask,
                                                  unsigned long long* word, uint32_t* bits) {
    const uint64_t z = mix64(g ^ 0xD6E8FEB86659FD93ull);
    *word = z & occ_mask;
    *bits = (1u << (uint32_t)((z >> 52) & 31u)) | (1u << (uint32_t)((z >> 58) & 31u));
}

// Coordinate of the cell with linear id L along dimension lane_id() for the
// lanes below k: the warp pays one 64-bit division per lane, and the other
// dimensions are fetched with shuffles, instead of k divisions per thread.
__device__ __forceinline__ uint32_t lane_cell_coord(const HjGrid& g, unsigned long long L) {
    const uint32_t j = lane_id();
    if (j >= g.k) return 0u;
    const unsigned long long q = L / g.mult[j];
    return (j + 1 < g.k) ? (uint32_t)(q % g.n_cells[j]) : (uint32_t)q;
}

// Quotient of r by a stencil width w in {1, 2, 3} (widths are 3 except where
// the stencil is clamped at the grid's edge): no integer division instruction.
__device__ __forceinline__ uint32_t div_w(uint32_t r, uint32_t w) {
    return w == 3u ? (uint32_t)(((unsigned long long)r * 0xAAAAAAABull) >> 33) : (w == 2u ? r >> 1 : r);
}

// Stencil rows of a cell's box (per dimension j the cells lo[j] .. lo[j] + w[j] - 1;
// `rows` is the product of w[1..k-1]).  Row r covers, along dimension j >= 1,
// coordinate lo[j] + the j-th mixed-radix digit of r (radices w[1], w[2], ...,
// dimension 1 fastest) and, along dimension 0, the w[0] cells from lo[0].
// A full box (every w[j] == 3 for j >= 1: the cell is not at the grid's upper
// edge) reads its rows' offsets from the grid's table; an edge box divides.
struct StencilRows {
    bool full;                  // offsets from grid.row_off
    unsigned long long first;   // linear id of row 0's first cell
};
__device__ __forceinline__ StencilRows stencil_rows(const HjGrid& g, const uint32_t* lo, uint32_t rows) {
    StencilRows s;
    s.full = g.row_off != nullptr && rows == g.full_rows;
    s.first = lo[0];
    for (uint32_t j = 1; j < g.k; ++j) s.first += (unsigned long long)lo[j] * g.mult[j];
    return s;
}
// Linear id of the first cell of row r (equal, modulo 2^64 like all linear-id
// arithmetic here, in both forms).
__device__ __forceinline__ unsigned long long stencil_row_id(const HjGrid& g, const StencilRows& s,
                                                             const uint32_t* lo, const uint32_t* w, uint32_t r) {
    if (s.full) return s.first + __ldg(g.row_off + r);
    uint32_t rem = r;
    unsigned long long id = lo[0];
    for (uint32_t j = 1; j < g.k; ++j) {
        const uint32_t qw = div_w(rem, w[j]);
        id += (unsigned long long)(lo[j] + (rem - qw * w[j])) * g.mult[j];
        rem = qw;
    }
    return id;
}

// The entry of group g: (first cell, id mask), or a zero mask when the group has
// no cell.  Probes stop at a free entry; the table is at most half full, so the
// loop ends after a few probes (and after capacity probes at the very most).
__device__ __forceinline__ uint2 group_find(const HjCellHash& h, unsigned long long g) {
    if (h.occ) {
        unsigned long long w;
        uint32_t b;
        occ_bits(g, h.occ_mask, &w, &b);
        if ((__ldg(h.occ + w) & b) != b) return make_uint2(kNoCell, 0u);
    }
    unsigned long long i = mix64(g) & h.mask;
    for (unsigned long long probe = 0; probe <= h.mask; ++probe) {
        const uint4 e = h.entries[i];
        const unsigned long long key = ((unsigned long long)e.y << 32) | e.x;
        if (key == g) return make_uint2(e.z, e.w);
        if (key == kEmptyLid) break;
        i = (i + 1) & h.mask;
    }
    return make_uint2(kNoCell, 0u);
}

// Points of the existing cells with linear ids lo .. lo + w - 1 (consecutive
// along dimension 0, w <= 4): one contiguous span [x, y) of the cell-ordered
// points, because the non-empty cells are sorted by linear id.
__device__ __forceinline__ uint2 cell_span(const HjCellHash& h, const uint32_t* cell_start, unsigned long long lo,
                                           uint32_t w) {
    const unsigned long long hi = lo + w - 1;
    uint32_t first = kNoCell, last = kNoCell;
    for (unsigned long long g = lo >> 2; g <= (hi >> 2); ++g) {
        const uint2 e = group_find(h, g);
        const uint32_t b0 = g == (lo >> 2) ? (uint32_t)(lo & 3u) : 0u;
        const uint32_t b1 = g == (hi >> 2) ? (uint32_t)(hi & 3u) : 3u;
        const uint32_t m = e.y & ((2u << b1) - 1u) & ~((1u << b0) - 1u);   // the group's ids in [lo, hi]
        if (m == 0u) continue;
        const uint32_t f = e.x + __popc(e.y & ((1u << (__ffs(m) - 1)) - 1u));
        const uint32_t l = e.x + __popc(e.y & ((2u << (31 - __clz(m))) - 1u)) - 1u;
        if (first == kNoCell) first = f;
        last = l;
    }
    if (first == kNoCell) return make_uint2(0u, 0u);
    return make_uint2(cell_start[first], cell_start[last + 1]);
}

}  // namespace hj
