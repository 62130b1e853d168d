// A caller written against the reference's interface only (the algorithm-0
// sequence of main.cu:89-273): it computes the grid geometry the way
// main.cu:449-520 does, then calls gridIndexingGPU, sortByWorkLoad and
// distanceTableNDGridBatches -- here resolved by hegjoin_b200's compatibility
// shim -- and writes the neighbour table as per-query sorted lists.
//
// usage: compat_main dataset eps out.bin
//   dataset: u32 n, u32 d, u32 sizeof(value), then n*d values; or, when the
//   name ends in ".txt", the reference's text format, read with importNDDataset
//   (main.cu:89) as main does.
//   out.bin: u64 totalNeighbors, u64 totalCandidates, u32 nNonEmptyCells,
//            (n + 1) u64 offsets, neighbour ids (u32).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "params.h"
#include "structs.h"
#include "hegjoin_compat.h"

int main(int argc, char** argv) {
    if (argc != 4) { fprintf(stderr, "usage: %s dataset eps out.bin\n", argv[0]); return 1; }
    std::string name = argv[1];
    unsigned int DBSIZE = 0;
    std::vector<DTYPE> db;
    if (name.size() > 4 && name.compare(name.size() - 4, 4, ".txt") == 0) {
        std::vector<std::vector<DTYPE> > pts;
        importNDDataset(&pts, argv[1]);
        DBSIZE = (unsigned int)pts.size();
        for (const auto& p : pts) db.insert(db.end(), p.begin(), p.end());
    } else {
        FILE* f = fopen(argv[1], "rb");
        if (!f) { perror(argv[1]); return 1; }
        uint32_t hdr[3];
        if (fread(hdr, 4, 3, f) != 3 || hdr[1] != GPUNUMDIM || hdr[2] != sizeof(DTYPE)) { fprintf(stderr, "bad dataset\n"); return 1; }
        DBSIZE = hdr[0];
        db.resize((size_t)DBSIZE * GPUNUMDIM);
        if (fread(db.data(), sizeof(DTYPE), db.size(), f) != db.size()) { fprintf(stderr, "short read\n"); return 1; }
        fclose(f);
    }
    DTYPE epsilon = atof(argv[2]);

    // grid geometry as main.cu:449-520 computes it
    DTYPE minArr[NUMINDEXEDDIM], maxArr[NUMINDEXEDDIM];
    unsigned int nCells[NUMINDEXEDDIM];
    for (int j = 0; j < NUMINDEXEDDIM; ++j) minArr[j] = maxArr[j] = db[j];
    for (unsigned i = 1; i < DBSIZE; ++i)
        for (int j = 0; j < NUMINDEXEDDIM; ++j) {
            DTYPE v = db[(size_t)i * GPUNUMDIM + j];
            if (v < minArr[j]) minArr[j] = v;
            if (v > maxArr[j]) maxArr[j] = v;
        }
    for (int j = 0; j < NUMINDEXEDDIM; ++j) { minArr[j] -= epsilon; maxArr[j] += epsilon; }
    uint64_t totalCells = 1;
    for (int j = 0; j < NUMINDEXEDDIM; ++j) {
        nCells[j] = (unsigned int)ceil((maxArr[j] - minArr[j]) / epsilon);
        totalCells *= nCells[j];
    }

    struct grid* index;
    struct gridCellLookup* gridCellLookupArr;
    unsigned int* indexLookupArr = new unsigned int[DBSIZE];
    DTYPE *dev_epsilon, *dev_database, *dev_minArr;
    struct grid* dev_index;
    unsigned int *dev_indexLookupArr, *dev_nCells, *dev_nNonEmptyCells;
    struct gridCellLookup* dev_gridCellLookupArr;
    unsigned int nNonEmptyCells = 0;
    gridIndexingGPU(&DBSIZE, totalCells, db.data(), &dev_database, &epsilon, &dev_epsilon, minArr, &dev_minArr,
                    &index, &dev_index, indexLookupArr, &dev_indexLookupArr, &gridCellLookupArr,
                    &dev_gridCellLookupArr, &nNonEmptyCells, &dev_nNonEmptyCells, nCells, &dev_nCells);

    neighborTableLookup* neighborTable = new neighborTableLookup[DBSIZE]();
    std::vector<struct neighborDataPtrs> pointersToNeighbors;
    unsigned int *originPointIndex, *dev_originPointIndex;
    uint64_t totalNeighbors = 0, totalCandidates = 0;
    struct schedulingCell* sortedDatabaseTmp;
    float staticPartition = 1.0;
    sortByWorkLoad(SM_GPU, &DBSIZE, &staticPartition, &totalCandidates, &sortedDatabaseTmp, &epsilon, &dev_epsilon,
                   db.data(), &dev_database, index, &dev_index, indexLookupArr, &dev_indexLookupArr,
                   gridCellLookupArr, &dev_gridCellLookupArr, minArr, &dev_minArr, nCells, &dev_nCells,
                   &nNonEmptyCells, &dev_nNonEmptyCells, &originPointIndex, &dev_originPointIndex);
    unsigned int nbQueriesGPU = 0;
    distanceTableNDGridBatches(SM_GPU, staticPartition, &DBSIZE, &epsilon, dev_epsilon, db.data(), dev_database, index,
                               dev_index, indexLookupArr, dev_indexLookupArr, gridCellLookupArr,
                               dev_gridCellLookupArr, minArr, dev_minArr, nCells, dev_nCells, &nNonEmptyCells,
                               dev_nNonEmptyCells, originPointIndex, dev_originPointIndex, neighborTable,
                               &pointersToNeighbors, &totalNeighbors, &nbQueriesGPU);
    printf("[RESULT] ~ Total result set size: %lu\n", (unsigned long)totalNeighbors);

    std::vector<uint64_t> off(DBSIZE + 1, 0);
    for (unsigned q = 0; q < DBSIZE; ++q) {
        const neighborTableLookup& e = neighborTable[q];
        off[q + 1] = off[q] + ((e.dataPtr && e.indexmax > e.indexmin) ? (uint64_t)(e.indexmax - e.indexmin) : 0);
    }
    std::vector<uint32_t> vals(off[DBSIZE]);
    for (unsigned q = 0; q < DBSIZE; ++q) {
        const neighborTableLookup& e = neighborTable[q];
        for (int i = e.indexmin; off[q + 1] > off[q] && i < e.indexmax; ++i) vals[off[q] + (i - e.indexmin)] = e.dataPtr[i];
        std::sort(vals.begin() + off[q], vals.begin() + off[q + 1]);
    }
    FILE* g = fopen(argv[3], "wb");
    fwrite(&totalNeighbors, 8, 1, g);
    fwrite(&totalCandidates, 8, 1, g);
    fwrite(&nNonEmptyCells, 4, 1, g);
    fwrite(off.data(), 8, off.size(), g);
    if (!vals.empty()) fwrite(vals.data(), 4, vals.size(), g);
    fclose(g);

    // caller-side frees, main.cu:416-443
    delete[] index; delete[] sortedDatabaseTmp; delete[] gridCellLookupArr; delete[] indexLookupArr;
    delete[] neighborTable; delete[] originPointIndex;
    for (auto& p : pointersToNeighbors) delete[] p.dataPtr;
    cudaFree(dev_epsilon); cudaFree(dev_database); cudaFree(dev_index); cudaFree(dev_indexLookupArr);
    cudaFree(dev_gridCellLookupArr); cudaFree(dev_minArr); cudaFree(dev_nCells); cudaFree(dev_nNonEmptyCells);
    cudaFree(dev_originPointIndex);
    return 0;
}
