// hj_internal.h -- library-internal structures shared by the .cu files.
#pragma once

#include "hj_common.cuh"

// Grid parameters passed by value to kernels.
struct HjGrid {
    uint32_t k;
    uint32_t n_cells[hj::kMaxK];
    unsigned long long mult[hj::kMaxK];   // mixed-radix multipliers, dimension 0 fastest
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
    uint32_t tc_kpad = 0;
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

}  // namespace hj
