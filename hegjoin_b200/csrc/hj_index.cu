// hj_index.cu -- grid geometry, grid-index build and workload order.
//
// Reference counterparts:
//   generateNDGridDimensions   main.cu:449-520
//   gridIndexingGPU            GPU.cu:74-398 (kernelIndexComputeNonemptyCells kernel.cu:34-66)
//   sortByWorkLoad             SortByWorkload.cu:19-247 (sortByWorkLoadGlobal kernel.cu:74-144)
//
// B200 design: everything stays on the device.  Cell ids are computed once,
// (cell id, point id) pairs are radix-sorted on only the bits totalCells
// needs, the non-empty-cell table comes from a run-boundary scan instead of the
// reference's device->host copy and host loop (GPU.cu:293-324), and the
// points are gathered into cell order so the refine kernels stream each
// cell's points as one contiguous range.  The workload pass resolves each
// cell's 3^k stencil once per cell as 3^(k-1) contiguous point ranges (the
// cells along dimension 0 are consecutive linear ids), one warp per cell.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <limits>
#include <map>
#include <mutex>

#include "hj_internal.h"

namespace hj {

// ---- error state ----------------------------------------------------------------
static thread_local char g_err[1024] = "";
void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
static std::atomic<uint64_t> g_launches{0};
static thread_local uint64_t t_launches = 0;
void count_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    ++t_launches;
}
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
uint64_t thread_launch_count() { return t_launches; }

static thread_local Workspace* t_workspace = nullptr;
Workspace* current_workspace() { return t_workspace; }
void set_current_workspace(Workspace* ws) { t_workspace = ws; }

static std::atomic<int64_t> g_fail_alloc_in{0};
bool injected_alloc_failure_armed() { return g_fail_alloc_in.load(std::memory_order_relaxed) > 0; }
bool injected_alloc_failure() {
    if (g_fail_alloc_in.load(std::memory_order_relaxed) <= 0) return false;
    return g_fail_alloc_in.fetch_sub(1, std::memory_order_relaxed) == 1;
}

hj_status ensure_smem_ptr(const void* kern, size_t bytes) {
    static std::mutex mu;
    static std::map<const void*, size_t> done;
    if (bytes <= 48 * 1024) return HJ_OK;
    std::lock_guard<std::mutex> lk(mu);
    size_t& have = done[kern];
    if (bytes <= have) return HJ_OK;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
        set_error("cudaFuncSetAttribute(%zu bytes): %s", bytes, cudaGetErrorString(e));
        return HJ_ERR_CUDA;
    }
    have = bytes;
    return HJ_OK;
}

void init_memory_pool() {
    static std::atomic<bool> done{false};
    if (done.exchange(true)) return;
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // Concurrent joins (the serving loop's workers) allocate and free on their own
        // streams.  By default the pool may hand one stream memory another stream freed
        // by making the allocation wait for that stream, which couples the requests;
        // reuse only memory whose free has completed, or that was freed on the same stream.
        int no = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    }
    cudaGetLastError();
}

template <typename T>
static T sq_threshold_t(T eps) {
    // sqrt is correctly rounded and monotone, so {x : RN(sqrt(x)) <= eps} is
    // {x <= T}; walk from RN(eps^2) to its largest member.
    T x = eps * eps;
    while (x > T(0) && std::sqrt(x) > eps) x = std::nextafter(x, T(0));
    while (true) {
        T nx = std::nextafter(x, std::numeric_limits<T>::infinity());
        if (std::sqrt(nx) <= eps) x = nx; else break;
    }
    return x;
}
double sq_threshold(double eps, int dtype) {
    if (dtype == HJ_F32) return (double)sq_threshold_t<float>((float)eps);
    return sq_threshold_t<double>(eps);
}

namespace {

template <typename T>
struct GeoT {
    T min_arr[kMaxK];
    T eps;
};

// kernel.cu:56 / kernel.cu:779: (unsigned)((x - minArr) / eps), IEEE ops in T.
__device__ __forceinline__ uint32_t cell_coord(float x, float mn, float eps) {
    return __float2uint_rz(__fdiv_rn(__fsub_rn(x, mn), eps));
}
__device__ __forceinline__ uint32_t cell_coord(double x, double mn, double eps) {
    return __double2uint_rz(__ddiv_rn(__dsub_rn(x, mn), eps));
}

// ---- geometry: per-dimension min / max ----------------------------------------------
template <typename T>
__global__ void k_minmax(const T* __restrict__ db, uint32_t n, uint32_t d, uint32_t k, T* out_min, T* out_max) {
    // per block: the minimum and maximum of each of the k indexed dimensions, all
    // dimensions in one launch (partials [dim][block])
    __shared__ T smin[32], smax[32];
    for (uint32_t j = 0; j < k; ++j) {
        T mn = db[j], mx = db[j];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (uint64_t)gridDim.x * blockDim.x) {
            T v = db[i * d + j];
            mn = v < mn ? v : mn;
            mx = v > mx ? v : mx;
        }
        for (int o = 16; o > 0; o >>= 1) {
            T a = __shfl_down_sync(0xffffffffu, mn, o), b = __shfl_down_sync(0xffffffffu, mx, o);
            mn = a < mn ? a : mn;
            mx = b > mx ? b : mx;
        }
        if (lane_id() == 0) { smin[threadIdx.x >> 5] = mn; smax[threadIdx.x >> 5] = mx; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                mn = smin[w] < mn ? smin[w] : mn;
                mx = smax[w] > mx ? smax[w] : mx;
            }
            out_min[(size_t)j * gridDim.x + blockIdx.x] = mn;
            out_max[(size_t)j * gridDim.x + blockIdx.x] = mx;
        }
        __syncthreads();
    }
}

template <typename T>
hj_status geometry_t(const T* db, uint32_t n, uint32_t d, uint32_t k, T eps, double* h_min, double* h_max,
                     uint32_t* h_ncells, uint64_t* h_total, cudaStream_t st) {
    const int blocks = std::min<int>(num_sms() * 4, std::max<uint32_t>(1, (n + 255) / 256));
    Scratch tmp(st);
    T* part = nullptr;
    HJ_TRY(tmp.alloc(&part, (size_t)2 * blocks * k));
    k_minmax<T><<<blocks, 256, 0, st>>>(db, n, d, k, part, part + (size_t)k * blocks);
    HJ_LAUNCHED();
    std::vector<T> hp((size_t)2 * blocks * k);
    HJ_CUDA(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(T), cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    uint64_t total = 1;
    for (uint32_t j = 0; j < k; ++j) {
        T mn = hp[(size_t)j * blocks], mx = hp[(size_t)(k + j) * blocks];
        for (int b = 1; b < blocks; ++b) {
            mn = std::min(mn, hp[(size_t)j * blocks + b]);
            mx = std::max(mx, hp[(size_t)(k + j) * blocks + b]);
        }
        // main.cu:489-509, in T
        T mnA = mn - eps;
        T mxA = mx + eps;
        T r = (mxA - mnA) / eps;
        uint32_t nc = (uint32_t)std::ceil(r);
        if (h_min) h_min[j] = (double)mnA;
        if (h_max) h_max[j] = (double)mxA;
        if (h_ncells) h_ncells[j] = nc;
        total *= nc;
    }
    if (h_total) *h_total = total;
    return HJ_OK;
}

// ---- index build -----------------------------------------------------------------------
template <typename T>
__global__ void k_cell_ids(const T* __restrict__ db, uint32_t n, uint32_t d, GeoT<T> geo, HjGrid grid,
                           unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* alias) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long lid = 0;
    bool al = false;
    for (uint32_t j = 0; j < grid.k; ++j) {
        uint32_t c = cell_coord(db[(uint64_t)i * d + j], geo.min_arr[j], geo.eps);
        al |= c >= grid.n_cells[j];
        lid += (unsigned long long)c * grid.mult[j];
    }
    keys[i] = lid;
    vals[i] = i;
    if (al) atomicExch(alias, 1u);
}

__global__ void k_run_flags(const unsigned long long* __restrict__ keys, uint32_t n, uint32_t* __restrict__ flags) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_cells(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ flags,
                        const uint32_t* __restrict__ pos, uint32_t n, unsigned long long* __restrict__ cell_lid,
                        uint32_t* __restrict__ cell_start, uint32_t* n_cells_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) {
        cell_lid[pos[i]] = keys[i];
        cell_start[pos[i]] = i;
    }
    if (i == n - 1) {
        uint32_t nc = pos[i] + flags[i];
        cell_start[nc] = n;
        *n_cells_out = nc;
    }
}

template <typename T>
__global__ void k_gather_rows(const T* __restrict__ db, const uint32_t* __restrict__ perm, uint32_t n, uint32_t d,
                              T* __restrict__ out) {
    uint64_t total = (uint64_t)n * d;
    for (uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; f < total; f += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = f / d, l = f - i * d;
        out[f] = db[(uint64_t)perm[i] * d + l];
    }
}

// ---- workload ------------------------------------------------------------------------
}  // namespace

// Per non-empty cell: number of candidates in its stencil (kernel.cu:74-144).
// One warp per cell; rows of the stencil (tuples over dimensions 1..k-1) are
// split over the lanes, each row being one contiguous range of linear ids.
__global__ void k_cell_workload(const unsigned long long* __restrict__ cell_lid, const uint32_t* __restrict__ cell_start,
                                uint32_t nC, HjGrid grid, HjCellHash hash, uint32_t* __restrict__ cell_nb,
                                unsigned long long* __restrict__ cell_work) {
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= nC) return;
    unsigned long long L = cell_lid[warp];
    uint32_t lo[kMaxK], w[kMaxK];
    uint32_t rows = 1;
    bool empty = false;
    const uint32_t cl = lane_cell_coord(grid, L);
    for (uint32_t j = 0; j < grid.k; ++j) {
        const uint32_t c = __shfl_sync(0xffffffffu, cl, j);
        uint32_t l = c - 1u;                                   // wraps at 0 (kernel.cu:113)
        uint32_t h = min(grid.n_cells[j] - 1u, c + 1u);        // kernel.cu:114
        if (l > h) empty = true;
        lo[j] = l;
        w[j] = h - l + 1;
        if (j > 0) rows *= w[j];
    }
    unsigned long long cnt = 0;
    if (!empty) {
        const StencilRows sr = stencil_rows(grid, lo, rows);
        for (uint32_t r = lane_id(); r < rows; r += 32) {
            const uint2 sp = cell_span(hash, cell_start, stencil_row_id(grid, sr, lo, w, r), w[0]);
            cnt += sp.y - sp.x;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane_id() == 0) {
        cell_nb[warp] = (uint32_t)cnt;
        cell_work[warp] = cnt * (unsigned long long)(cell_start[warp + 1] - cell_start[warp]);
    }
}

namespace {

__global__ void k_desc_keys(const uint32_t* __restrict__ nb, uint32_t nC, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    keys[i] = ~nb[i];     // ascending order of the complement = descending candidates
    vals[i] = i;
}

__global__ void k_max_u32(const uint32_t* __restrict__ a, uint32_t n, uint32_t* out) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, a[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if (lane_id() == 0) atomicMax(out, m);
}

__global__ void k_block_counts(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cell_start, uint32_t nC,
                               uint32_t qb, uint32_t* __restrict__ cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    uint32_t c = order[i];
    uint32_t pop = cell_start[c + 1] - cell_start[c];
    cnt[i] = (pop + qb - 1) / qb;
}

__global__ void k_make_blocks(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cell_start,
                              const uint32_t* __restrict__ cell_nb, const uint32_t* __restrict__ off, uint32_t nC,
                              uint32_t qb, HjBlock* __restrict__ blocks) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    uint32_t c = order[i];
    uint32_t s = cell_start[c], e = cell_start[c + 1];
    uint32_t o = off[i];
    for (uint32_t q = s; q < e; q += qb, ++o) blocks[o] = HjBlock{c, q, min(e, q + qb), cell_nb[c]};
}

__global__ void k_origin_index(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cell_start,
                               const uint32_t* __restrict__ perm, const uint32_t* __restrict__ off, uint32_t nC,
                               uint32_t* __restrict__ out) {
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= nC) return;
    uint32_t c = order[warp];
    uint32_t s = cell_start[c], e = cell_start[c + 1], o = off[warp];
    for (uint32_t q = s + lane_id(); q < e; q += 32) out[o + (q - s)] = perm[q];
}

__global__ void k_pop_in_order(const uint32_t* __restrict__ order, const uint32_t* __restrict__ cell_start, uint32_t nC,
                               uint32_t* __restrict__ pop) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    uint32_t c = order[i];
    pop[i] = cell_start[c + 1] - cell_start[c];
}

__global__ void k_export_index(const unsigned long long* __restrict__ cell_lid, const uint32_t* __restrict__ cell_start,
                               uint32_t nC, hj_grid_cell_lookup* lookup, hj_grid* grid) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    if (lookup) lookup[i] = hj_grid_cell_lookup{i, 0u, cell_lid[i]};
    if (grid) grid[i] = hj_grid{(int32_t)cell_start[i], (int32_t)cell_start[i + 1] - 1};
}

__global__ void k_export_sched(const uint32_t* __restrict__ order, const uint32_t* __restrict__ nb, uint32_t nC,
                               hj_scheduling_cell* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    uint32_t c = order[i];
    out[i] = hj_scheduling_cell{(int32_t)nb[c], (int32_t)c};
}

template <typename T>
hj_status index_create_t(const T* d_db, uint32_t n, uint32_t d, uint32_t k, T eps, const double* h_min,
                         const uint32_t* h_ncells, cudaStream_t st, hj_index* ix) {
    ix->n = n; ix->d = d; ix->k = k;
    ix->eps = (double)eps;
    ix->thr = sq_threshold((double)eps, ix->dtype);
    GeoT<T> geo{};
    geo.eps = eps;
    ix->grid.k = k;
    unsigned long long mul = 1;
    ix->total_cells = 1;
    for (uint32_t j = 0; j < k; ++j) {
        geo.min_arr[j] = (T)h_min[j];
        ix->min_arr[j] = (double)geo.min_arr[j];
        ix->grid.n_cells[j] = h_ncells[j];
        ix->grid.mult[j] = mul;
        mul *= h_ncells[j];
        ix->total_cells *= h_ncells[j];
    }
    // temporaries: freed on every return path; the index's own arrays are freed by free_index on failure
    Scratch tmp(st);
    unsigned long long *keys = nullptr, *keys_tmp = nullptr;
    uint32_t *vals_tmp = nullptr, *flags = nullptr, *pos = nullptr, *scalars = nullptr;
    HJ_TRY(tmp.alloc(&keys, n));
    HJ_TRY(tmp.alloc(&keys_tmp, n));
    HJ_TRY(dalloc(&ix->perm, n, st));
    HJ_TRY(tmp.alloc(&vals_tmp, n));
    HJ_TRY(tmp.alloc(&scalars, 4));
    HJ_CUDA(cudaMemsetAsync(scalars, 0, 4 * sizeof(uint32_t), st));
    unsigned grid1 = (n + 255) / 256;
    k_cell_ids<T><<<grid1, 256, 0, st>>>(d_db, n, d, geo, ix->grid, keys, ix->perm, scalars);
    HJ_LAUNCHED();
    uint32_t nbits = bits_for(ix->total_cells > 0 ? ix->total_cells - 1 : 0);
    HJ_TRY(radix_sort_u64_u32(reinterpret_cast<uint64_t*>(keys), ix->perm, reinterpret_cast<uint64_t*>(keys_tmp),
                              vals_tmp, n, nbits, st));
    tmp.release(keys_tmp);
    tmp.release(vals_tmp);
    HJ_TRY(tmp.alloc(&flags, n));
    HJ_TRY(tmp.alloc(&pos, n));
    k_run_flags<<<grid1, 256, 0, st>>>(keys, n, flags);
    HJ_LAUNCHED();
    HJ_CUDA(cudaMemcpyAsync(pos, flags, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    HJ_TRY(scan_u32_inplace(pos, n, st));
    HJ_TRY(dalloc(&ix->cell_lid, (size_t)n, st));
    HJ_TRY(dalloc(&ix->cell_start, (size_t)n + 1, st));
    k_cells<<<grid1, 256, 0, st>>>(keys, flags, pos, n, ix->cell_lid, ix->cell_start, scalars + 1);
    HJ_LAUNCHED();
    T* pts = nullptr;
    HJ_TRY(dalloc(&pts, (size_t)n * d, st));
    ix->pts = pts;
    unsigned grid2 = (unsigned)std::min<uint64_t>(((uint64_t)n * d + 255) / 256, (uint64_t)num_sms() * 16);
    k_gather_rows<T><<<grid2, 256, 0, st>>>(d_db, ix->perm, n, d, pts);
    HJ_LAUNCHED();
    uint32_t hs[2];
    HJ_CUDA(cudaMemcpyAsync(hs, scalars, sizeof(hs), cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    ix->aliasing = hs[0];
    ix->nC = hs[1];
    if (ix->aliasing) {
        set_error("grid aliasing: a point's cell coordinate reaches nCells in some indexed dimension "
                  "(epsilon below the coordinates' rounding granularity); unsupported");
        return HJ_ERR_UNSUPPORTED;
    }
    return HJ_OK;
}

// The first cell of each group inserts the group's entry: key, first cell, mask
// of the group's ids (its cells are the next ones in the table, at most four).
// The key word pair is claimed with a 64-bit compare-and-swap on the entry's
// first 8 bytes; first cell and mask are written after it.
__global__ void k_hash_insert(const unsigned long long* __restrict__ lid, uint32_t nC, uint4* entries,
                              unsigned long long mask, uint32_t* occ, unsigned long long occ_mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nC) return;
    const unsigned long long g = lid[i] >> 2;
    if (i > 0 && (lid[i - 1] >> 2) == g) return;
    uint32_t m = 0;
    for (uint32_t j = i; j < nC && j < i + 4 && (lid[j] >> 2) == g; ++j) m |= 1u << (uint32_t)(lid[j] & 3u);
    if (occ) {
        unsigned long long w;
        uint32_t b;
        occ_bits(g, occ_mask, &w, &b);
        atomicOr(occ + w, b);
    }
    unsigned long long s = mix64(g) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {   // the table is at most half full
        unsigned long long* kw = reinterpret_cast<unsigned long long*>(&entries[s]);
        const unsigned long long prev = atomicCAS(kw, kEmptyLid, g);
        if (prev == kEmptyLid) {
            entries[s].z = i;
            entries[s].w = m;
            return;
        }
        s = (s + 1) & mask;
    }
}

// The grid's row-offset table (HjGrid::row_off), for k <= kRowOffMaxK.
__global__ void k_row_offsets(HjGrid g, unsigned long long* off) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.full_rows) return;
    uint32_t rem = r;
    unsigned long long o = 0;
    for (uint32_t j = 1; j < g.k; ++j) {
        o += (unsigned long long)(rem % 3u) * g.mult[j];
        rem /= 3u;
    }
    off[r] = o;
}

hj_status build_row_offsets(hj_index* ix, cudaStream_t st) {
    if (ix->grid.k == 0 || ix->grid.k > kRowOffMaxK) return HJ_OK;
    uint32_t rows = 1;
    for (uint32_t j = 1; j < ix->grid.k; ++j) rows *= 3;
    HJ_TRY(dalloc(&ix->row_off, rows, st));
    ix->grid.full_rows = rows;
    k_row_offsets<<<(rows + 255) / 256, 256, 0, st>>>(ix->grid, ix->row_off);
    HJ_LAUNCHED();
    ix->grid.row_off = ix->row_off;
    return HJ_OK;
}

// Smallest table (entries) that gets an occupancy filter: 32 MB of entries.
constexpr unsigned long long kOccMinCap = 1ull << 21;

// The cell hash of an index whose cell table is built (capacity: the power of
// two at least twice the number of cells, an upper bound on the groups that
// needs no count from the device, at least 64).  From kOccMinCap entries on, an
// occupancy filter of capacity / 4 words (16 bits per cell, a sixteenth of the
// table's bytes) goes with it.
hj_status build_cell_hash(hj_index* ix, cudaStream_t st) {
    unsigned long long cap = 64;
    while (cap < 2ull * ix->nC) cap <<= 1;
    HJ_TRY(dalloc(&ix->hash_entries, (size_t)cap, st));
    HJ_CUDA(cudaMemsetAsync(ix->hash_entries, 0xFF, (size_t)cap * sizeof(uint4), st));
    ix->hash_mask = cap - 1;
    if (cap >= kOccMinCap) {
        HJ_TRY(dalloc(&ix->hash_occ, (size_t)(cap / 4), st));
        HJ_CUDA(cudaMemsetAsync(ix->hash_occ, 0, (size_t)cap, st));
        ix->occ_mask = cap / 4 - 1;
    }
    if (ix->nC) {
        k_hash_insert<<<(ix->nC + 255) / 256, 256, 0, st>>>(ix->cell_lid, ix->nC, ix->hash_entries, ix->hash_mask,
                                                           ix->hash_occ, ix->occ_mask);
        HJ_LAUNCHED();
    }
    return HJ_OK;
}

void free_index(hj_index* ix, cudaStream_t st) {
    tc_release(ix);
    dfree(ix->hash_entries, st);
    dfree(ix->hash_occ, st);
    dfree(ix->row_off, st);
    ix->grid.row_off = nullptr;
    ix->grid.full_rows = 0;
    dfree(ix->pts, st);
    dfree(ix->perm, st);
    dfree(ix->cell_lid, st);
    dfree(ix->cell_start, st);
    dfree(ix->cell_nb, st);
    dfree(ix->cell_order, st);
    dfree(ix->tc_a, st);
    dfree(ix->tc_b, st);
    dfree(ix->tc_err, st);
    dfree(ix->tc_pband, st);
}

}  // namespace

hj_status build_blocks(const hj_index* ix, uint32_t qb, HjBlock** d_blocks, uint32_t* n_blocks, cudaStream_t st) {
    uint32_t nC = ix->nC;
    Scratch tmp(st);
    uint32_t* cnt = nullptr;
    HJ_TRY(tmp.alloc(&cnt, (size_t)nC + 1));
    unsigned g = (nC + 255) / 256;
    k_block_counts<<<g, 256, 0, st>>>(ix->cell_order, ix->cell_start, nC, qb, cnt);
    HJ_LAUNCHED();
    HJ_CUDA(cudaMemsetAsync(cnt + nC, 0, 4, st));
    HJ_TRY(scan_u32_inplace(cnt, (uint64_t)nC + 1, st));
    uint32_t nb = 0;
    HJ_CUDA(cudaMemcpyAsync(&nb, cnt + nC, 4, cudaMemcpyDeviceToHost, st));
    HJ_CUDA(cudaStreamSynchronize(st));
    HjBlock* blocks = nullptr;
    HJ_TRY(tmp.alloc_pool(&blocks, (size_t)std::max<uint32_t>(nb, 1)));   // handed to the caller
    k_make_blocks<<<g, 256, 0, st>>>(ix->cell_order, ix->cell_start, ix->cell_nb, cnt, nC, qb, blocks);
    HJ_LAUNCHED();
    *d_blocks = tmp.keep(blocks);
    *n_blocks = nb;
    return HJ_OK;
}

}  // namespace hj

using namespace hj;

extern "C" {

const char* hj_last_error(void) { return hj::g_err; }

void hj_debug_fail_alloc(uint64_t nth) { hj::g_fail_alloc_in.store((int64_t)nth, std::memory_order_relaxed); }

hj_status hj_debug_pool_used(uint64_t* bytes) {
    if (!bytes) { set_error("hj_debug_pool_used: null argument"); return HJ_ERR_INVALID; }
    int dev = 0;
    cudaMemPool_t pool;
    HJ_CUDA(cudaGetDevice(&dev));
    HJ_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    unsigned long long used = 0;   // cudaMemPoolAttrUsedMemCurrent is a 64-bit count
    HJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    *bytes = (uint64_t)used;
    return HJ_OK;
}
hj_status hj_debug_pool_peak(uint64_t* bytes, int reset) {
    if (!bytes) { set_error("hj_debug_pool_peak: null argument"); return HJ_ERR_INVALID; }
    int dev = 0;
    cudaMemPool_t pool;
    HJ_CUDA(cudaGetDevice(&dev));
    HJ_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    unsigned long long high = 0;
    HJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &high));
    *bytes = (uint64_t)high;
    if (reset) {
        unsigned long long zero = 0;   // resets the high-water mark to the current use
        HJ_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
    }
    return HJ_OK;
}
const char* hj_version(void) { return "hegjoin_b200 0.1 (sm_100a)"; }
uint64_t hj_kernel_launch_count(void) { return hj::launch_count(); }

hj_status hj_grid_geometry(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype, double eps,
                           double* h_min_arr, double* h_max_arr, uint32_t* h_n_cells, uint64_t* h_total_cells,
                           void* stream) {
    if (!d_db || n == 0 || d == 0 || k == 0 || k > (uint32_t)kMaxK || k > d || !(eps > 0)) {
        set_error("hj_grid_geometry: invalid arguments (n=%u d=%u k=%u eps=%g)", n, d, k, eps);
        return HJ_ERR_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    if (dtype == HJ_F32)
        return geometry_t<float>((const float*)d_db, n, d, k, (float)eps, h_min_arr, h_max_arr, h_n_cells,
                                 h_total_cells, st);
    if (dtype == HJ_F64)
        return geometry_t<double>((const double*)d_db, n, d, k, eps, h_min_arr, h_max_arr, h_n_cells, h_total_cells,
                                  st);
    set_error("hj_grid_geometry: unknown dtype %d", dtype);
    return HJ_ERR_INVALID;
}

hj_status hj_index_create(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype, double eps,
                          const double* h_min_arr, const uint32_t* h_n_cells, void* stream, hj_index** out) {
    if (!out) { set_error("hj_index_create: null out"); return HJ_ERR_INVALID; }
    *out = nullptr;
    if (!d_db || n == 0 || d == 0 || d > (uint32_t)kMaxD || k == 0 || k > (uint32_t)kMaxK || k > d || !(eps > 0) ||
        (dtype != HJ_F32 && dtype != HJ_F64) || n >= 0x7FFFFFFFu) {
        set_error("hj_index_create: invalid arguments (n=%u d=%u k=%u dtype=%d eps=%g)", n, d, k, dtype, eps);
        return HJ_ERR_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    double mn[kMaxK], mx[kMaxK];
    uint32_t nc[kMaxK];
    if (!h_min_arr || !h_n_cells) {
        HJ_TRY(hj_grid_geometry(d_db, n, d, k, dtype, eps, mn, mx, nc, nullptr, stream));
        h_min_arr = mn;
        h_n_cells = nc;
    }
    uint64_t tot = 1;
    for (uint32_t j = 0; j < k; ++j) {
        if (h_n_cells[j] == 0) { set_error("hj_index_create: nCells[%u] == 0", j); return HJ_ERR_INVALID; }
        if (tot > ~0ull / h_n_cells[j]) { set_error("hj_index_create: totalCells overflows 64 bits"); return HJ_ERR_UNSUPPORTED; }
        tot *= h_n_cells[j];
    }
    init_memory_pool();
    hj_index* ix = new hj_index();
    ix->dtype = dtype;
    ix->stream = st;
    cudaGetDevice(&ix->device);
    hj_status s = (dtype == HJ_F32)
                      ? index_create_t<float>((const float*)d_db, n, d, k, (float)eps, h_min_arr, h_n_cells, st, ix)
                      : index_create_t<double>((const double*)d_db, n, d, k, eps, h_min_arr, h_n_cells, st, ix);
    // linear ids are below totalCells <= 2^64 - 1, so none equals the hash's free-slot mark
    if (s == HJ_OK) s = build_cell_hash(ix, st);
    if (s == HJ_OK) s = build_row_offsets(ix, st);
    if (s != HJ_OK) {
        free_index(ix, st);
        cudaStreamSynchronize(st);
        delete ix;
        return s;
    }
    *out = ix;
    return HJ_OK;
}

hj_status hj_index_destroy(hj_index* ix) {
    if (!ix) return HJ_OK;
    // stream-ordered frees on the index's own stream: no device-wide synchronisation,
    // so concurrent joins on other streams keep running
    free_index(ix, ix->stream);
    delete ix;
    return HJ_OK;
}

hj_status hj_index_get_info(const hj_index* ix, hj_index_info* o) {
    if (!ix || !o) { set_error("hj_index_get_info: null argument"); return HJ_ERR_INVALID; }
    *o = hj_index_info{};
    o->n = ix->n; o->d = ix->d; o->k = ix->k; o->dtype = (uint32_t)ix->dtype;
    o->n_nonempty_cells = ix->nC;
    o->grid_aliasing = ix->aliasing;
    o->total_cells = ix->total_cells;
    o->total_candidates = ix->total_candidates;
    o->eps = ix->eps;
    o->sq_threshold = ix->thr;
    for (uint32_t j = 0; j < ix->k; ++j) {
        o->min_arr[j] = ix->min_arr[j];
        o->n_cells[j] = ix->grid.n_cells[j];
    }
    return HJ_OK;
}

hj_status hj_index_export(const hj_index* ix, hj_grid_cell_lookup* d_lookup, hj_grid* d_grid, uint32_t* d_index_lookup,
                          void* stream) {
    if (!ix) { set_error("hj_index_export: null index"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    if (d_lookup || d_grid) {
        k_export_index<<<(ix->nC + 255) / 256, 256, 0, st>>>(ix->cell_lid, ix->cell_start, ix->nC, d_lookup, d_grid);
        HJ_LAUNCHED();
    }
    if (d_index_lookup)
        HJ_CUDA(cudaMemcpyAsync(d_index_lookup, ix->perm, (size_t)ix->n * 4, cudaMemcpyDeviceToDevice, st));
    return HJ_OK;
}

hj_status hj_index_views(const hj_index* ix, const void** pts, const uint32_t** perm, const uint64_t** cell_lid,
                         const uint32_t** cell_start) {
    if (!ix) { set_error("hj_index_views: null index"); return HJ_ERR_INVALID; }
    if (pts) *pts = ix->pts;
    if (perm) *perm = ix->perm;
    if (cell_lid) *cell_lid = reinterpret_cast<const uint64_t*>(ix->cell_lid);
    if (cell_start) *cell_start = ix->cell_start;
    return HJ_OK;
}

hj_status hj_sort_by_workload(hj_index* ix, void* stream, uint64_t* total_candidates) {
    if (!ix) { set_error("hj_sort_by_workload: null index"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    if (!ix->have_workload) {
        uint32_t nC = ix->nC;
        // a previous attempt that failed part-way may have left these allocated
        dfree(ix->cell_nb, st);
        dfree(ix->cell_order, st);
        Scratch tmp(st);
        unsigned long long* work = nullptr;
        uint32_t *keys = nullptr, *keys_tmp = nullptr, *vals_tmp = nullptr, *dmax = nullptr;
        uint64_t* dsum = nullptr;
        HJ_TRY(dalloc(&ix->cell_nb, nC, st));
        HJ_TRY(tmp.alloc(&work, nC));
        unsigned g = (unsigned)(((uint64_t)nC * 32 + 255) / 256);
        k_cell_workload<<<g, 256, 0, st>>>(ix->cell_lid, ix->cell_start, nC, ix->grid, cell_hash(ix), ix->cell_nb,
                                           work);
        HJ_LAUNCHED();
        HJ_TRY(tmp.alloc(&dsum, 1));
        HJ_TRY(reduce_sum_u64(reinterpret_cast<uint64_t*>(work), nC, dsum, st));
        HJ_TRY(tmp.alloc(&dmax, 1));
        HJ_CUDA(cudaMemsetAsync(dmax, 0, 4, st));
        k_max_u32<<<std::min<unsigned>((nC + 255) / 256, num_sms() * 4), 256, 0, st>>>(ix->cell_nb, nC, dmax);
        HJ_LAUNCHED();
        HJ_TRY(tmp.alloc(&keys, nC));
        HJ_TRY(tmp.alloc(&keys_tmp, nC));
        HJ_TRY(tmp.alloc(&vals_tmp, nC));
        HJ_TRY(dalloc(&ix->cell_order, nC, st));
        k_desc_keys<<<(nC + 255) / 256, 256, 0, st>>>(ix->cell_nb, nC, keys, ix->cell_order);
        HJ_LAUNCHED();
        HJ_TRY(radix_sort_u32_u32(keys, ix->cell_order, keys_tmp, vals_tmp, nC, 32, st));
        uint64_t tot = 0;
        HJ_CUDA(cudaMemcpyAsync(&tot, dsum, 8, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaMemcpyAsync(&ix->max_nb, dmax, 4, cudaMemcpyDeviceToHost, st));
        HJ_CUDA(cudaStreamSynchronize(st));
        ix->total_candidates = tot;
        ix->have_workload = true;
    }
    if (total_candidates) *total_candidates = ix->total_candidates;
    return HJ_OK;
}

hj_status hj_workload_export(const hj_index* ix, hj_scheduling_cell* d_sched, uint32_t* d_origin, void* stream) {
    if (!ix || !ix->have_workload) { set_error("hj_workload_export: run hj_sort_by_workload first"); return HJ_ERR_INVALID; }
    cudaStream_t st = as_stream(stream);
    uint32_t nC = ix->nC;
    if (d_sched) {
        k_export_sched<<<(nC + 255) / 256, 256, 0, st>>>(ix->cell_order, ix->cell_nb, nC, d_sched);
        HJ_LAUNCHED();
    }
    if (d_origin) {
        Scratch tmp(st);
        uint32_t* off = nullptr;
        HJ_TRY(tmp.alloc(&off, nC));
        k_pop_in_order<<<(nC + 255) / 256, 256, 0, st>>>(ix->cell_order, ix->cell_start, nC, off);
        HJ_LAUNCHED();
        HJ_TRY(scan_u32_inplace(off, nC, st));
        k_origin_index<<<(unsigned)(((uint64_t)nC * 32 + 255) / 256), 256, 0, st>>>(ix->cell_order, ix->cell_start,
                                                                                   ix->perm, off, nC, d_origin);
        HJ_LAUNCHED();
    }
    return HJ_OK;
}

}  // extern "C"
