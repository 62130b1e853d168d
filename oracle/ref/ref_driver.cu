// ref_driver.cu -- TEST INFRASTRUCTURE ONLY: runs the reference's own GPU-only
// join (algorithm 0) on a binary dataset and dumps what it computed, so the
// CPU oracle and the CUDA path can be checked against the reference itself.
//
// It replays the caller sequence of main.cu:89-273 for searchMode 0 --
// generateNDGridDimensions, gridIndexingGPU, sortByWorkLoad,
// distanceTableNDGridBatches -- calling the reference's compiled functions
// (linked from its own objects, see oracle/ref/Makefile), then walks the
// reference's neighborTable (structs.h:35-41; indexmax is exclusive,
// GPU.cu:1767) into per-query sorted neighbour lists.
//
// usage: ref_driver <dataset.bin> <eps> <out_prefix>
//   dataset.bin: u32 n, u32 d, u32 sizeof(value), then n*d values, row-major.
// outputs: <out_prefix>.geom.bin, .index.bin, .sched.bin, .pairs.bin and one
// JSON summary line on stdout (prefixed by "HJREF ").

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <string>
#include <vector>

#include <omp.h>

#include "params.h"
#include "structs.h"
#include "main.h"
#include "GPU.h"
#include "SortByWorkload.h"
#include "WorkQueue.h"

template <typename V>
static void put(FILE* f, const V* p, size_t n) {
    if (n && fwrite(p, sizeof(V), n, f) != n) { perror("write"); exit(2); }
}

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s dataset.bin eps out_prefix\n", argv[0]);
        return 1;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 1; }
    uint32_t hdr[3];
    if (fread(hdr, 4, 3, f) != 3) { fprintf(stderr, "bad header\n"); return 1; }
    const uint32_t n = hdr[0], d = hdr[1], vs = hdr[2];
    if (d != GPUNUMDIM || vs != sizeof(DTYPE)) {
        fprintf(stderr, "dataset is %u-D with %u-byte values; this build is %d-D with %zu-byte DTYPE\n", d, vs,
                GPUNUMDIM, sizeof(DTYPE));
        return 1;
    }
    std::vector<DTYPE> flat((size_t)n * d);
    if (fread(flat.data(), sizeof(DTYPE), flat.size(), f) != flat.size()) { fprintf(stderr, "short read\n"); return 1; }
    fclose(f);

    // main.cu:56 -- DTYPE epsilon = atof(argv[EPSILON_ARG])
    DTYPE epsilon = atof(argv[2]);
    std::vector<std::vector<DTYPE> > NDdataPoints(n, std::vector<DTYPE>(d));
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < d; ++j) NDdataPoints[i][j] = flat[(size_t)i * d + j];
    unsigned int DBSIZE = n;
    setQueueIndexCPU(DBSIZE);
    DTYPE* database = new DTYPE[(size_t)DBSIZE * GPUNUMDIM];
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < d; ++j) database[(size_t)i * GPUNUMDIM + j] = NDdataPoints[i][j];
    float staticPartition = 1.0;

    DTYPE* minArr = new DTYPE[NUMINDEXEDDIM];
    DTYPE* maxArr = new DTYPE[NUMINDEXEDDIM];
    unsigned int* nCells = new unsigned int[NUMINDEXEDDIM];
    uint64_t totalCells = 0;
    unsigned int nNonEmptyCells = 0;
    generateNDGridDimensions(&NDdataPoints, epsilon, minArr, maxArr, nCells, &totalCells);

    struct grid* index;
    struct gridCellLookup* gridCellLookupArr;
    unsigned int* indexLookupArr = new unsigned int[n];
    DTYPE *dev_epsilon, *dev_database, *dev_minArr;
    struct grid* dev_index;
    unsigned int *dev_indexLookupArr, *dev_nCells, *dev_nNonEmptyCells;
    struct gridCellLookup* dev_gridCellLookupArr;

    double t0 = omp_get_wtime();
    gridIndexingGPU(&DBSIZE, totalCells, database, &dev_database, &epsilon, &dev_epsilon, minArr, &dev_minArr, &index,
                    &dev_index, indexLookupArr, &dev_indexLookupArr, &gridCellLookupArr, &dev_gridCellLookupArr,
                    &nNonEmptyCells, &dev_nNonEmptyCells, nCells, &dev_nCells);
    double t1 = omp_get_wtime();

    neighborTableLookup* neighborTable = new neighborTableLookup[n]();   // entries never written stay empty
    std::vector<struct neighborDataPtrs> pointersToNeighbors;
    unsigned int* originPointIndex;
    unsigned int* dev_originPointIndex;
    uint64_t totalNeighbors = 0, totalCandidates = 0;
    struct schedulingCell* sortedDatabaseTmp;
    sortByWorkLoad(SM_GPU, &DBSIZE, &staticPartition, &totalCandidates, &sortedDatabaseTmp, &epsilon, &dev_epsilon,
                   database, &dev_database, index, &dev_index, indexLookupArr, &dev_indexLookupArr, gridCellLookupArr,
                   &dev_gridCellLookupArr, minArr, &dev_minArr, nCells, &dev_nCells, &nNonEmptyCells,
                   &dev_nNonEmptyCells, &originPointIndex, &dev_originPointIndex);
    double t2 = omp_get_wtime();
    unsigned int nbQueriesGPU = 0;
    distanceTableNDGridBatches(SM_GPU, staticPartition, &DBSIZE, &epsilon, dev_epsilon, database, dev_database, index,
                               dev_index, indexLookupArr, dev_indexLookupArr, gridCellLookupArr,
                               dev_gridCellLookupArr, minArr, dev_minArr, nCells, dev_nCells, &nNonEmptyCells,
                               dev_nNonEmptyCells, originPointIndex, dev_originPointIndex, neighborTable,
                               &pointersToNeighbors, &totalNeighbors, &nbQueriesGPU);
    double t3 = omp_get_wtime();

    std::string pre = argv[3];
    {
        FILE* g = fopen((pre + ".geom.bin").c_str(), "wb");
        put(g, minArr, NUMINDEXEDDIM);
        put(g, nCells, NUMINDEXEDDIM);
        put(g, &totalCells, 1);
        fclose(g);
    }
    {
        FILE* g = fopen((pre + ".index.bin").c_str(), "wb");
        put(g, &nNonEmptyCells, 1);
        std::vector<uint64_t> lid(nNonEmptyCells);
        std::vector<uint32_t> idx(nNonEmptyCells);
        std::vector<int32_t> gmin(nNonEmptyCells), gmax(nNonEmptyCells);
        for (unsigned c = 0; c < nNonEmptyCells; ++c) {
            lid[c] = gridCellLookupArr[c].gridLinearID;
            idx[c] = gridCellLookupArr[c].idx;
            gmin[c] = index[c].indexmin;
            gmax[c] = index[c].indexmax;
        }
        put(g, lid.data(), lid.size());
        put(g, idx.data(), idx.size());
        put(g, gmin.data(), gmin.size());
        put(g, gmax.data(), gmax.size());
        put(g, indexLookupArr, n);
        fclose(g);
    }
    {
        FILE* g = fopen((pre + ".sched.bin").c_str(), "wb");
        put(g, &totalCandidates, 1);
        for (unsigned c = 0; c < nNonEmptyCells; ++c) {
            int32_t v[2] = {sortedDatabaseTmp[c].nbPoints, sortedDatabaseTmp[c].cellId};
            put(g, v, 2);
        }
        put(g, originPointIndex, n);
        fclose(g);
    }
    uint64_t table_sum = 0;
    {
        std::vector<uint64_t> off(n + 1, 0);
        for (uint32_t q = 0; q < n; ++q) {
            const neighborTableLookup& e = neighborTable[q];
            uint64_t c = (e.dataPtr && e.indexmax > e.indexmin) ? (uint64_t)(e.indexmax - e.indexmin) : 0;
            off[q + 1] = off[q] + c;
        }
        table_sum = off[n];
        std::vector<uint32_t> vals(table_sum);
        for (uint32_t q = 0; q < n; ++q) {
            const neighborTableLookup& e = neighborTable[q];
            if (off[q + 1] == off[q]) continue;
            for (int i = e.indexmin; i < e.indexmax; ++i) vals[off[q] + (i - e.indexmin)] = (uint32_t)e.dataPtr[i];
            std::sort(vals.begin() + off[q], vals.begin() + off[q + 1]);
        }
        FILE* g = fopen((pre + ".pairs.bin").c_str(), "wb");
        put(g, &totalNeighbors, 1);
        put(g, &table_sum, 1);
        put(g, off.data(), off.size());
        put(g, vals.data(), vals.size());
        fclose(g);
    }
    printf("HJREF {\"n\": %u, \"d\": %u, \"k\": %d, \"dtype_bytes\": %zu, \"eps\": %.17g, \"total_cells\": %llu, "
           "\"nonempty_cells\": %u, \"total_candidates\": %llu, \"total_neighbors\": %llu, \"table_pairs\": %llu, "
           "\"batches\": %zu, \"queries_gpu\": %u, \"s_index\": %.6f, \"s_sort\": %.6f, \"s_join\": %.6f}\n",
           n, d, NUMINDEXEDDIM, sizeof(DTYPE), (double)epsilon, (unsigned long long)totalCells, nNonEmptyCells,
           (unsigned long long)totalCandidates, (unsigned long long)totalNeighbors, (unsigned long long)table_sum,
           pointersToNeighbors.size(), nbQueriesGPU, t1 - t0, t2 - t1, t3 - t2);
    return 0;
}
