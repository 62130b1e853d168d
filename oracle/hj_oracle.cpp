// hj_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of HEGJoin's GPU-only self-join (algorithm 0), used as the
// parity checker for the CUDA path in hegjoin_b200/.  Nothing in the product
// links or calls this file; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg load it (through oracle/__init__.py).
//
// Parity status: pinned against the reference itself, built from its own
// sources by oracle/ref/Makefile (sm_100a, with the cell-lookup comparison made
// callable on the device) and run by oracle/ref/ref_driver.cu; the golden
// fixtures it produced live in
// tests/golden/ and tests/test_oracle_golden.py checks this file against them.
//
// Every routine cites the reference file:line whose arithmetic it restates.
// The arithmetic is done in the dataset's type T (float or double) exactly as
// the reference's device code does it: IEEE single/double operations in the
// order the source writes them, correctly rounded division and sqrt, and the
// squared-distance accumulation contracted to fma(diff, diff, acc) the way
// nvcc's default --fmad=true compiles kernel.cu:350-353 (the alternative,
// uncontracted order is kept behind `fma_mode == 0` for the contraction probe).
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>

namespace {

// kernel.cu:310-325 / main.cu:740-754: mixed radix, dimension 0 fastest.
inline uint64_t linear_id(const uint32_t* idx, const uint32_t* nCells, uint32_t k) {
    uint64_t off = 0, mul = 1;
    for (uint32_t i = 0; i < k; ++i) {
        off += (uint64_t)idx[i] * mul;
        mul *= nCells[i];
    }
    return off;
}

// kernel.cu:56 and kernel.cu:779: (unsigned)((x - minArr) / eps) in T.
template <typename T>
inline uint32_t cell_coord(T x, T mn, T eps) {
    T a = x - mn;
    T c = a / eps;
    return (uint32_t)c;
}

// kernel.cu:780-781 call CUDA's max(int, unsigned) overload, which compares
// as unsigned: max(0, c - 1) is therefore c - 1 itself, and for coordinate 0
// it wraps to UINT_MAX, which leaves that dimension's loop empty.
inline uint32_t box_lo(uint32_t c) { return c - 1u; }
inline uint32_t box_hi(uint32_t c, uint32_t n) { return std::min(n - 1u, c + 1u); }

template <typename T>
inline T sqdist(const T* c, const T* q, uint32_t d, int fma_mode) {
    // kernel.cu:350-353: acc += (c_l - q_l) * (c_l - q_l), l = 0..d-1.
    T acc = 0;
    if (fma_mode) {
        for (uint32_t l = 0; l < d; ++l) {
            T diff = c[l] - q[l];
            acc = std::fma(diff, diff, acc);
        }
    } else {
        for (uint32_t l = 0; l < d; ++l) {
            T diff = c[l] - q[l];
            T sq = diff * diff;
            acc = acc + sq;
        }
    }
    return acc;
}

struct Index {
    std::vector<uint64_t> cell_lid;   // sorted unique linear ids (gridCellLookupArr[i].gridLinearID)
    std::vector<int32_t> first, last; // grid[i] = {indexmin, indexmax} (inclusive)
    std::vector<uint32_t> lookup;     // indexLookupArr
};

template <typename T>
void build_index(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, const T* minArr,
                 const uint32_t* nCells, Index& ix) {
    // GPU.cu:239-324: cell id per point, stable sort of (lid, id), run scan.
    std::vector<uint64_t> lid(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint32_t idx[32];
        for (uint32_t j = 0; j < k; ++j) idx[j] = cell_coord<T>(db[(size_t)i * d + j], minArr[j], eps);
        lid[i] = linear_id(idx, nCells, k);
    }
    ix.lookup.resize(n);
    for (uint32_t i = 0; i < n; ++i) ix.lookup[i] = i;
    std::stable_sort(ix.lookup.begin(), ix.lookup.end(),
                     [&](uint32_t a, uint32_t b) { return lid[a] < lid[b]; });
    ix.cell_lid.clear(); ix.first.clear(); ix.last.clear();
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t L = lid[ix.lookup[i]];
        if (i == 0 || L != ix.cell_lid.back()) {
            if (i) ix.last.push_back((int32_t)i - 1);
            ix.cell_lid.push_back(L);
            ix.first.push_back((int32_t)i);
        }
    }
    if (n) ix.last.push_back((int32_t)n - 1);
}

inline int64_t find_cell(const Index& ix, uint64_t L) {
    auto it = std::lower_bound(ix.cell_lid.begin(), ix.cell_lid.end(), L);
    if (it == ix.cell_lid.end() || *it != L) return -1;
    return it - ix.cell_lid.begin();
}

// Enumerate the 3^k stencil of a point (kernel.cu:775-789 + kernelloops.h),
// calling f(cell_index) for every non-empty cell, in the reference's loop order
// (dimension 0 outermost).
template <typename T, typename F>
void for_each_stencil_cell(const T* p, uint32_t k, T eps, const T* minArr, const uint32_t* nCells,
                           const Index& ix, F&& f) {
    uint32_t lo[32], hi[32], cur[32];
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t c = cell_coord<T>(p[i], minArr[i], eps);
        lo[i] = box_lo(c);
        hi[i] = box_hi(c, nCells[i]);
        if (lo[i] > hi[i]) return;  // empty range in one dimension: no cells at all
    }
    for (uint32_t i = 0; i < k; ++i) cur[i] = lo[i];
    while (true) {
        int64_t ci = find_cell(ix, linear_id(cur, nCells, k));
        if (ci >= 0) f(ci);
        // odometer, last dimension innermost
        int32_t j = (int32_t)k - 1;
        while (j >= 0) {
            if (cur[j] < hi[j]) { ++cur[j]; break; }
            cur[j] = lo[j];
            --j;
        }
        if (j < 0) break;
    }
}

// import_dataset.cpp:10-40 (importNDDataset), restated with the same standard
// library calls: tokens from getline(in, f, ','), values from a stringstream
// over each token with `>>` until an extraction fails.  Writes at most
// `capacity` values to out and returns how many the file holds.
template <typename T>
uint64_t import_text(const char* path, T* out, uint64_t capacity) {
    std::ifstream in(path);
    uint64_t cnt = 0;
    for (std::string f; std::getline(in, f, ',');) {
        T v;
        std::stringstream ss(f);
        while (ss >> v) {
            if (cnt < capacity) out[cnt] = v;
            ++cnt;
            if (ss.peek() == ',') ss.ignore();
        }
    }
    return cnt;
}
inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

// main.cu:449-520 (generateNDGridDimensions), arithmetic in T.
#define HJO_GEOM(T, SUF)                                                                        \
    void hjo_geometry_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, T* minArr,   \
                            T* maxArr, uint32_t* nCells, uint64_t* totalCells) {                 \
        for (uint32_t j = 0; j < k; ++j) { minArr[j] = db[j]; maxArr[j] = db[j]; }               \
        for (uint32_t i = 1; i < n; ++i)                                                         \
            for (uint32_t j = 0; j < k; ++j) {                                                   \
                T v = db[(size_t)i * d + j];                                                     \
                if (v < minArr[j]) minArr[j] = v;                                                \
                if (v > maxArr[j]) maxArr[j] = v;                                                \
            }                                                                                    \
        for (uint32_t j = 0; j < k; ++j) { minArr[j] -= eps; maxArr[j] += eps; }                 \
        for (uint32_t j = 0; j < k; ++j) {                                                       \
            T r = (maxArr[j] - minArr[j]) / eps;                                                 \
            nCells[j] = (uint32_t)std::ceil(r);                                                  \
        }                                                                                        \
        uint64_t t = nCells[0];                                                                  \
        for (uint32_t j = 1; j < k; ++j) t *= nCells[j];                                         \
        *totalCells = t;                                                                         \
    }
HJO_GEOM(float, f32)
HJO_GEOM(double, f64)

// GPU.cu:74-398 (gridIndexingGPU): outputs gridCellLookupArr ids, grid
// first/last (inclusive) and indexLookupArr.  Returns nNonEmptyCells.
#define HJO_INDEX(T, SUF)                                                                          \
    uint32_t hjo_index_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, const T* minArr,\
                             const uint32_t* nCells, uint64_t* cell_lid, int32_t* first,           \
                             int32_t* last, uint32_t* lookup) {                                    \
        Index ix;                                                                                  \
        build_index<T>(db, n, d, k, eps, minArr, nCells, ix);                                      \
        size_t nc = ix.cell_lid.size();                                                            \
        std::memcpy(cell_lid, ix.cell_lid.data(), nc * 8);                                         \
        std::memcpy(first, ix.first.data(), nc * 4);                                               \
        std::memcpy(last, ix.last.data(), nc * 4);                                                 \
        std::memcpy(lookup, ix.lookup.data(), (size_t)n * 4);                                      \
        return (uint32_t)nc;                                                                       \
    }
HJO_INDEX(float, f32)
HJO_INDEX(double, f64)

// kernel.cu:74-144 (sortByWorkLoadGlobal): per non-empty cell, in cell order,
// the summed population of the non-empty cells in the stencil of the cell's
// first point.  Returns totalCandidates as SortByWorkload.cu:155-217 sums it.
#define HJO_WORK(T, SUF)                                                                            \
    uint64_t hjo_cell_workload_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps,          \
                                     const T* minArr, const uint32_t* nCells, uint32_t* nbPoints) {  \
        Index ix;                                                                                   \
        build_index<T>(db, n, d, k, eps, minArr, nCells, ix);                                       \
        int64_t nc = (int64_t)ix.cell_lid.size();                                                   \
        uint64_t total = 0;                                                                         \
        _Pragma("omp parallel for schedule(dynamic, 64) reduction(+ : total)")                      \
        for (int64_t c = 0; c < nc; ++c) {                                                          \
            const T* p = db + (size_t)ix.lookup[ix.first[c]] * d;                                   \
            uint32_t cnt = 0;                                                                       \
            for_each_stencil_cell<T>(p, k, eps, minArr, nCells, ix, [&](int64_t ci) {               \
                cnt += (uint32_t)(ix.last[ci] - ix.first[ci] + 1);                                  \
            });                                                                                     \
            nbPoints[c] = cnt;                                                                      \
            total += (uint64_t)cnt * (uint64_t)(ix.last[c] - ix.first[c] + 1);                      \
        }                                                                                           \
        return total;                                                                               \
    }
HJO_WORK(float, f32)
HJO_WORK(double, f64)

// kernel.cu:727-802 with evaluateCell (378-412) and evalPoint (333-370):
// for every query point q (by original id) and every candidate c in q's
// stencil cells, emit (q, c) when sqrt(d2) <= eps.  Two passes: counts, then
// neighbour ids (each list sorted ascending).  `counts` has n entries;
// `offsets` (n + 1) and `vals` may be null for the count-only pass.
#define HJO_JOIN(T, SUF)                                                                             \
    uint64_t hjo_join_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, const T* minArr,  \
                            const uint32_t* nCells, int fma_mode, uint32_t* counts,                  \
                            const uint64_t* offsets, uint32_t* vals) {                               \
        Index ix;                                                                                    \
        build_index<T>(db, n, d, k, eps, minArr, nCells, ix);                                        \
        uint64_t total = 0;                                                                          \
        _Pragma("omp parallel for schedule(dynamic, 16) reduction(+ : total)")                       \
        for (int64_t q = 0; q < (int64_t)n; ++q) {                                                   \
            const T* p = db + (size_t)q * d;                                                         \
            uint64_t w = offsets ? offsets[q] : 0;                                                   \
            uint32_t cnt = 0;                                                                        \
            for_each_stencil_cell<T>(p, k, eps, minArr, nCells, ix, [&](int64_t ci) {                \
                for (int32_t s = ix.first[ci]; s <= ix.last[ci]; ++s) {                              \
                    uint32_t cid = ix.lookup[s];                                                     \
                    T acc = sqdist<T>(db + (size_t)cid * d, p, d, fma_mode);                         \
                    if (std::sqrt(acc) <= eps) {                                                     \
                        if (vals) vals[w + cnt] = cid;                                               \
                        ++cnt;                                                                       \
                    }                                                                                \
                }                                                                                    \
            });                                                                                      \
            if (vals) std::sort(vals + w, vals + w + cnt);                                           \
            counts[q] = cnt;                                                                         \
            total += cnt;                                                                            \
        }                                                                                            \
        return total;                                                                                \
    }
HJO_JOIN(float, f32)
HJO_JOIN(double, f64)

// The join restricted to a sample of query ids (the timed CPU baseline):
// returns the number of pairs the sampled queries emit.
#define HJO_JOIN_SAMPLE(T, SUF)                                                                      \
    uint64_t hjo_join_sample_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps,            \
                                   const T* minArr, const uint32_t* nCells, const uint32_t* qids,    \
                                   uint32_t nq, double* seconds) {                                    \
        Index ix;                                                                                    \
        build_index<T>(db, n, d, k, eps, minArr, nCells, ix);                                        \
        double t0 = omp_get_wtime();                                                                 \
        uint64_t total = 0;                                                                          \
        _Pragma("omp parallel for schedule(dynamic, 1) reduction(+ : total)")                        \
        for (int64_t s = 0; s < (int64_t)nq; ++s) {                                                  \
            const T* p = db + (size_t)qids[s] * d;                                                   \
            uint64_t cnt = 0;                                                                        \
            for_each_stencil_cell<T>(p, k, eps, minArr, nCells, ix, [&](int64_t ci) {                \
                for (int32_t j = ix.first[ci]; j <= ix.last[ci]; ++j) {                              \
                    T acc = sqdist<T>(db + (size_t)ix.lookup[j] * d, p, d, 1);                       \
                    cnt += std::sqrt(acc) <= eps;                                                    \
                }                                                                                    \
            });                                                                                      \
            total += cnt;                                                                            \
        }                                                                                            \
        *seconds = omp_get_wtime() - t0;                                                             \
        return total;                                                                                \
    }
HJO_JOIN_SAMPLE(float, f32)
HJO_JOIN_SAMPLE(double, f64)

// The join's neighbour lists for a sample of query ids (kernel.cu:727-802, as
// hjo_join): counts[s] for query qids[s], and, when the lists fit `capacity`,
// the lists themselves (each sorted ascending) concatenated in sample order.
// Returns the total list length; the caller re-calls with a larger buffer when
// it exceeds `capacity` (vals is then left untouched).
#define HJO_JOIN_LISTS(T, SUF)                                                                       \
    uint64_t hjo_join_lists_##SUF(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps,             \
                                  const T* minArr, const uint32_t* nCells, const uint32_t* qids,     \
                                  uint32_t nq, uint32_t* counts, uint32_t* vals, uint64_t capacity) { \
        Index ix;                                                                                    \
        build_index<T>(db, n, d, k, eps, minArr, nCells, ix);                                        \
        std::vector<std::vector<uint32_t>> lists(nq);                                                \
        _Pragma("omp parallel for schedule(dynamic, 1)")                                             \
        for (int64_t s = 0; s < (int64_t)nq; ++s) {                                                  \
            const T* p = db + (size_t)qids[s] * d;                                                   \
            std::vector<uint32_t>& L = lists[s];                                                     \
            for_each_stencil_cell<T>(p, k, eps, minArr, nCells, ix, [&](int64_t ci) {                \
                for (int32_t j = ix.first[ci]; j <= ix.last[ci]; ++j) {                              \
                    uint32_t cid = ix.lookup[j];                                                     \
                    T acc = sqdist<T>(db + (size_t)cid * d, p, d, 1);                                \
                    if (std::sqrt(acc) <= eps) L.push_back(cid);                                     \
                }                                                                                    \
            });                                                                                      \
            std::sort(L.begin(), L.end());                                                           \
        }                                                                                            \
        uint64_t total = 0;                                                                          \
        for (uint32_t s = 0; s < nq; ++s) {                                                          \
            counts[s] = (uint32_t)lists[s].size();                                                   \
            total += lists[s].size();                                                                \
        }                                                                                            \
        if (vals && total <= capacity) {                                                             \
            uint64_t w = 0;                                                                          \
            for (uint32_t s = 0; s < nq; ++s) {                                                      \
                std::memcpy(vals + w, lists[s].data(), lists[s].size() * 4);                         \
                w += lists[s].size();                                                                \
            }                                                                                        \
        }                                                                                            \
        return total;                                                                                \
    }
HJO_JOIN_LISTS(float, f32)
HJO_JOIN_LISTS(double, f64)

// The reference generator's text layout (datasets/dataset_gen_fixed_len_expo_dist.cpp:
// 76-83: "v, v, ..., v" per line) with `digits` significant digits per value, for
// ingest tests and timings.  Returns 0 on success.
int hjo_write_text(const char* path, const void* vals, uint64_t n, uint32_t d, int is_double, int digits) {
    FILE* f = std::fopen(path, "w");
    if (!f) return 1;
    std::vector<char> buf(1 << 20);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    for (uint64_t i = 0; i < n; ++i) {
        for (uint32_t j = 0; j < d; ++j) {
            const double v = is_double ? static_cast<const double*>(vals)[i * d + j]
                                       : (double)static_cast<const float*>(vals)[i * d + j];
            std::fprintf(f, j + 1 < d ? "%.*g, " : "%.*g\n", digits, v);
        }
    }
    return std::fclose(f) != 0;
}

uint64_t hjo_import_text_f32(const char* path, float* out, uint64_t capacity) {
    return import_text<float>(path, out, capacity);
}
uint64_t hjo_import_text_f64(const char* path, double* out, uint64_t capacity) {
    return import_text<double>(path, out, capacity);
}

// Squared distance of one pair in the reference order (for error statistics).
double hjo_sqdist_f32(const float* a, const float* b, uint32_t d, int fma_mode) {
    return (double)sqdist<float>(a, b, d, fma_mode);
}
double hjo_sqdist_f64(const double* a, const double* b, uint32_t d, int fma_mode) {
    return sqdist<double>(a, b, d, fma_mode);
}

// Order-independent per-query digest of a neighbour list: (count, sum of
// mix64(id), xor of mix64(id ^ salt)).  Used to compare pair sets that are too
// large to ship as lists.
void hjo_digest(const uint64_t* offsets, const uint32_t* vals, uint32_t n, uint64_t* sum_out,
                uint64_t* xor_out) {
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < (int64_t)n; ++q) {
        uint64_t s = 0, x = 0;
        for (uint64_t i = offsets[q]; i < offsets[q + 1]; ++i) {
            s += mix64(vals[i]);
            x ^= mix64((uint64_t)vals[i] ^ 0x5bd1e9955bd1e995ull);
        }
        sum_out[q] = s;
        xor_out[q] = x;
    }
}

// SortByWorkload.cu:97-98 orders the schedulingCell array (in cell order,
// cellId = cell index) with std::sort on nbPoints descending.  Replaying that
// exact call on the same input gives the reference's (implementation-defined)
// order among equal counts, which its batch estimator then depends on.
struct HjoSchedCell {
    int nbPoints;
    int cellId;
};
void hjo_ref_cell_order(const uint32_t* nbPoints, uint32_t ncells, int32_t* order_out) {
    std::vector<HjoSchedCell> v(ncells);
    for (uint32_t i = 0; i < ncells; ++i) v[i] = HjoSchedCell{(int)nbPoints[i], (int)i};
    std::sort(v.begin(), v.end(), [](const HjoSchedCell& a, const HjoSchedCell& b) { return a.nbPoints > b.nbPoints; });
    for (uint32_t i = 0; i < ncells; ++i) order_out[i] = v[i].cellId;
}

int hjo_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
