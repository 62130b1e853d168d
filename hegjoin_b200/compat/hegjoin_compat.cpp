// hegjoin_compat.cpp -- the reference's GPU-path entry points on top of the
// hegjoin_b200 C ABI.  Compile this file together with the caller's params.h
// and structs.h (it replaces GPU.cu, SortByWorkload.cu and kernel.cu) and link
// libhegjoin_b200.so and the CUDA runtime.
//
// Every function keeps the reference's signature, ownership rules
// (new[] / cudaMalloc for everything it hands back, main.cu:416-443) and its
// print-and-continue error convention; the work runs in the library.  The
// index handle is kept in a registry keyed by the device copy of the dataset,
// which every later call receives.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "hegjoin_b200.h"
#include "hegjoin_compat.h"

static_assert(sizeof(struct gridCellLookup) == sizeof(hj_grid_cell_lookup), "gridCellLookup layout");
static_assert(sizeof(struct grid) == sizeof(hj_grid), "grid layout");
static_assert(sizeof(struct schedulingCell) == sizeof(hj_scheduling_cell), "schedulingCell layout");

// The reference's work-queue hooks (WorkQueue.h); called when the caller links them.
void setQueueIndex(unsigned int index) __attribute__((weak));
void setMaxNeighbors(unsigned int maxNeighbors) __attribute__((weak));
void setWorkQueueReady() __attribute__((weak));

namespace {

std::mutex g_mu;
std::map<const void*, hj_index*> g_index;

constexpr int kDtype = sizeof(DTYPE) == 8 ? HJ_F64 : HJ_F32;

hj_index* lookup(const void* dev_database) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_index.find(dev_database);
    return it == g_index.end() ? nullptr : it->second;
}

bool report(const char* tag, hj_status s) {
    if (s == HJ_OK) return true;
    printf("[%s] ~ Error: hegjoin_b200 status %d: %s\n", tag, s, hj_last_error());
    fflush(stdout);
    return false;
}

bool report_cuda(const char* tag, const char* what, cudaError_t e) {
    if (e == cudaSuccess) return true;
    printf("[%s] ~ Error: %s -- error with code %d\n[%s] ~   Details: %s\n", tag, what, (int)e, tag,
           cudaGetErrorString(e));
    fflush(stdout);
    return false;
}

template <typename T>
bool dev_copy(const char* tag, T** dst, const T* src, size_t count) {
    if (!report_cuda(tag, "cudaMalloc", cudaMalloc((void**)dst, sizeof(T) * (count ? count : 1)))) return false;
    return report_cuda(tag, "cudaMemcpy", cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice));
}

}  // namespace

void gridIndexingGPU(unsigned int* DBSIZE, uint64_t totalCells, DTYPE* database, DTYPE** dev_database,
                     DTYPE* epsilon, DTYPE** dev_epsilon, DTYPE* minArr, DTYPE** dev_minArr, struct grid** index,
                     struct grid** dev_index, unsigned int* indexLookupArr, unsigned int** dev_indexLookupArr,
                     struct gridCellLookup** gridCellLookupArr, struct gridCellLookup** dev_gridCellLookupArr,
                     unsigned int* nNonEmptyCells, unsigned int** dev_nNonEmptyCells, unsigned int* nCells,
                     unsigned int** dev_nCells) {
    const char* T = "INDEX";
    const unsigned n = *DBSIZE;
    (void)totalCells;
    if (!dev_copy(T, dev_database, database, (size_t)n * GPUNUMDIM)) return;
    if (!dev_copy(T, dev_epsilon, epsilon, 1)) return;
    if (!dev_copy(T, dev_minArr, minArr, NUMINDEXEDDIM)) return;
    if (!dev_copy(T, dev_nCells, nCells, NUMINDEXEDDIM)) return;
    double mn[NUMINDEXEDDIM];
    for (int j = 0; j < NUMINDEXEDDIM; ++j) mn[j] = (double)minArr[j];
    hj_index* ix = nullptr;
    if (!report(T, hj_index_create(*dev_database, n, GPUNUMDIM, NUMINDEXEDDIM, kDtype, (double)*epsilon, mn, nCells,
                                   nullptr, &ix)))
        return;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_index[*dev_database] = ix;
    }
    hj_index_info info;
    hj_index_get_info(ix, &info);
    const unsigned nc = info.n_nonempty_cells;
    *nNonEmptyCells = nc;
    if (!dev_copy(T, dev_nNonEmptyCells, nNonEmptyCells, 1)) return;
    if (!report_cuda(T, "cudaMalloc", cudaMalloc((void**)dev_index, sizeof(struct grid) * nc))) return;
    if (!report_cuda(T, "cudaMalloc", cudaMalloc((void**)dev_gridCellLookupArr, sizeof(struct gridCellLookup) * nc)))
        return;
    if (!report_cuda(T, "cudaMalloc", cudaMalloc((void**)dev_indexLookupArr, sizeof(unsigned int) * n))) return;
    if (!report(T, hj_index_export(ix, reinterpret_cast<hj_grid_cell_lookup*>(*dev_gridCellLookupArr),
                                   reinterpret_cast<hj_grid*>(*dev_index), *dev_indexLookupArr, nullptr)))
        return;
    *index = new grid[nc];
    *gridCellLookupArr = new gridCellLookup[nc];
    report_cuda(T, "cudaMemcpy", cudaMemcpy(*index, *dev_index, sizeof(struct grid) * nc, cudaMemcpyDeviceToHost));
    report_cuda(T, "cudaMemcpy", cudaMemcpy(*gridCellLookupArr, *dev_gridCellLookupArr,
                                            sizeof(struct gridCellLookup) * nc, cudaMemcpyDeviceToHost));
    report_cuda(T, "cudaMemcpy", cudaMemcpy(indexLookupArr, *dev_indexLookupArr, sizeof(unsigned int) * n,
                                            cudaMemcpyDeviceToHost));
    printf("[INDEX] ~ Number of full cells (non-empty): %u\n", nc);
}

void sortByWorkLoad(unsigned int searchMode, unsigned int* DBSIZE, float* staticPartition, uint64_t* totalCandidates,
                    struct schedulingCell** sortedDatabaseTmp, DTYPE* epsilon, DTYPE** dev_epsilon, DTYPE* database,
                    DTYPE** dev_database, struct grid* index, struct grid** dev_index, unsigned int* indexLookupArr,
                    unsigned int** dev_indexLookupArr, struct gridCellLookup* gridCellLookupArr,
                    struct gridCellLookup** dev_gridCellLookupArr, DTYPE* minArr, DTYPE** dev_minArr,
                    unsigned int* nCells, unsigned int** dev_nCells, unsigned int* nNonEmptyCells,
                    unsigned int** dev_nNonEmptyCells, unsigned int** originPointIndex,
                    unsigned int** dev_originPointIndex) {
    const char* T = "SORT";
    (void)epsilon; (void)dev_epsilon; (void)database; (void)index; (void)dev_index; (void)indexLookupArr;
    (void)dev_indexLookupArr; (void)gridCellLookupArr; (void)dev_gridCellLookupArr; (void)minArr; (void)dev_minArr;
    (void)nCells; (void)dev_nCells; (void)dev_nNonEmptyCells;
    if (searchMode == SM_HYBRID_STATIC && !STATIC_SPLIT_QUERIES && staticPartition && *staticPartition == -1.0f)
        printf("[SORT] ~ Warning: the static CPU/GPU partition model (StaticPartition.cpp) is not provided; "
               "the GPU keeps all queries\n");
    hj_index* ix = lookup(*dev_database);
    if (!ix) { printf("[SORT] ~ Error: gridIndexingGPU was not called for this dataset\n"); return; }
    uint64_t tot = 0;
    if (!report(T, hj_sort_by_workload(ix, nullptr, &tot))) return;
    *totalCandidates = tot;
    const unsigned nc = *nNonEmptyCells, n = *DBSIZE;
    hj_scheduling_cell* d_sched = nullptr;
    if (!report_cuda(T, "cudaMalloc", cudaMalloc((void**)&d_sched, sizeof(hj_scheduling_cell) * (nc ? nc : 1))))
        return;
    if (!report_cuda(T, "cudaMalloc", cudaMalloc((void**)dev_originPointIndex, sizeof(unsigned int) * n))) return;
    if (!report(T, hj_workload_export(ix, d_sched, *dev_originPointIndex, nullptr))) return;
    *sortedDatabaseTmp = new schedulingCell[nc];
    *originPointIndex = new unsigned int[n];
    report_cuda(T, "cudaMemcpy", cudaMemcpy(*sortedDatabaseTmp, d_sched, sizeof(hj_scheduling_cell) * nc,
                                            cudaMemcpyDeviceToHost));
    report_cuda(T, "cudaMemcpy", cudaMemcpy(*originPointIndex, *dev_originPointIndex, sizeof(unsigned int) * n,
                                            cudaMemcpyDeviceToHost));
    cudaFree(d_sched);
    if (setMaxNeighbors && nc) setMaxNeighbors((unsigned)(*sortedDatabaseTmp)[0].nbPoints);
    if (setWorkQueueReady) setWorkQueueReady();
    printf("[SORT | RESULT] ~ Total number of candidate points to refine: %llu\n", (unsigned long long)tot);
}

void distanceTableNDGridBatches(int searchMode, float staticPartition, unsigned int* DBSIZE, DTYPE* epsilon,
                                DTYPE* dev_epsilon, DTYPE* database, DTYPE* dev_database, struct grid* index,
                                struct grid* dev_index, unsigned int* indexLookupArr, unsigned int* dev_indexLookupArr,
                                struct gridCellLookup* gridCellLookupArr, struct gridCellLookup* dev_gridCellLookupArr,
                                DTYPE* minArr, DTYPE* dev_minArr, unsigned int* nCells, unsigned int* dev_nCells,
                                unsigned int* nNonEmptyCells, unsigned int* dev_nNonEmptyCells,
                                unsigned int* originPointIndex, unsigned int* dev_originPointIndex,
                                struct neighborTableLookup* neighborTable,
                                std::vector<struct neighborDataPtrs>* pointersToNeighbors, uint64_t* totalNeighbors,
                                unsigned int* nbQueriesGPU) {
    const char* T = "GPU";
    (void)staticPartition; (void)epsilon; (void)dev_epsilon; (void)database; (void)index; (void)dev_index;
    (void)indexLookupArr; (void)dev_indexLookupArr; (void)gridCellLookupArr; (void)dev_gridCellLookupArr;
    (void)minArr; (void)dev_minArr; (void)nCells; (void)dev_nCells; (void)nNonEmptyCells; (void)dev_nNonEmptyCells;
    (void)originPointIndex; (void)dev_originPointIndex;
    *totalNeighbors = 0;
    if (searchMode != SM_GPU) {
        printf("[GPU] ~ Error: only the GPU-only join (search mode %d) is provided by hegjoin_b200\n", SM_GPU);
        return;
    }
    hj_index* ix = lookup(dev_database);
    if (!ix) { printf("[GPU] ~ Error: gridIndexingGPU was not called for this dataset\n"); return; }
    const unsigned n = *DBSIZE;
    hj_join_opts o;
    hj_join_opts_default(&o);
    // Each grouped batch comes to the host as it completes (GPU.cu:1542-1573): keys and
    // values through pinned staging, then a new int[] of values per batch and the
    // neighbour-table entries pointing into it.  Nothing stays on the device, so the
    // result may exceed device memory, as in the reference.
    struct Sink {
        neighborTableLookup* table;
        std::vector<neighborDataPtrs>* ptrs;
        int* keys = nullptr;
        int* vals = nullptr;
        uint64_t cap = 0;
        ~Sink() {
            if (keys) cudaFreeHost(keys);
            if (vals) cudaFreeHost(vals);
        }
        static hj_status on_batch(hj_batch_view* b, void* user, void* stream) {
            Sink* S = static_cast<Sink*>(user);
            if (b->count == 0) return HJ_OK;
            if (b->count > 0x7FFFFFFFull) return HJ_ERR_OVERFLOW;   // the table stores int offsets
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            if (b->count > S->cap) {
                if (S->keys) cudaFreeHost(S->keys);
                if (S->vals) cudaFreeHost(S->vals);
                S->keys = S->vals = nullptr;
                S->cap = 0;
                if (cudaMallocHost((void**)&S->keys, b->count * sizeof(int)) != cudaSuccess ||
                    cudaMallocHost((void**)&S->vals, b->count * sizeof(int)) != cudaSuccess)
                    return HJ_ERR_OOM;
                S->cap = b->count;
            }
            if (cudaMemcpyAsync(S->keys, b->d_keys, b->count * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaMemcpyAsync(S->vals, b->d_vals, b->count * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return HJ_ERR_CUDA;
            unsigned cnt = (unsigned)b->count;
            int* kept = new int[cnt];   // owned by pointersToNeighbors, as in the reference
            constructNeighborTableKeyValueWithPtrs(S->keys, S->vals, S->table, kept, &cnt);
            S->ptrs->push_back(neighborDataPtrs{kept, (int)cnt});
            return HJ_OK;
        }
    } sink;
    sink.table = neighborTable;
    sink.ptrs = pointersToNeighbors;
    hj_join_stats st;
    if (!report(T, hj_join_stream(ix, &o, &Sink::on_batch, &sink, nullptr, nullptr, nullptr, nullptr, &st))) return;
    if (setQueueIndex) setQueueIndex(n);   // all queries went to the GPU
    *totalNeighbors = st.total_pairs;
    *nbQueriesGPU = n;
    printf("[GPU] ~ Total result set size on host: %llu\n", (unsigned long long)st.total_pairs);
}

void constructNeighborTableKeyValueWithPtrs(int* pointIDKey, int* pointInDistValue,
                                            struct neighborTableLookup* neighborTable, int* pointersToNeighbors,
                                            unsigned int* cnt) {
    // GPU.cu:1731-1776: copy the values, then one table entry per run of equal
    // keys (indexmax exclusive).  The run scan stops at cnt - 1.
    const unsigned c = *cnt;
    std::memcpy(pointersToNeighbors, pointInDistValue, sizeof(int) * c);
    unsigned s = 0;
    for (unsigned i = 1; i <= c; ++i) {
        if (i == c || pointIDKey[i] != pointIDKey[i - 1]) {
            const int key = pointIDKey[s];
            neighborTable[key].pointID = key;
            neighborTable[key].indexmin = (int)s;
            neighborTable[key].indexmax = (int)i;
            neighborTable[key].dataPtr = pointersToNeighbors;
            s = i;
        }
    }
}

void warmUpGPU() { cudaFree(0); }
