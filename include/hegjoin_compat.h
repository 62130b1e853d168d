/* hegjoin_compat.h -- the reference's GPU-path entry points, unchanged.
 *
 * Declarations matching GPU.h:9-95 and SortByWorkload.h:7-30 of HEGJoin, so a
 * caller written against the reference (main.cu) links against
 * hegjoin_b200/compat/hegjoin_compat.cpp + libhegjoin_b200.so instead of
 * GPU.cu, SortByWorkload.cu and kernel.cu.  The shim is compiled with the
 * caller's own params.h (GPUNUMDIM, NUMINDEXEDDIM, DTYPE) and structs.h.
 *
 * Behavioural contract (kept from the reference): host out-arrays are
 * allocated with new[] and device arrays with cudaMalloc, the caller frees
 * them with delete[] / cudaFree (main.cu:416-443); errors are printed and
 * execution continues; only searchMode 0 (SM_GPU) is provided.
 */
#ifndef HEGJOIN_COMPAT_H
#define HEGJOIN_COMPAT_H

#include <cstdint>
#include <vector>

#include "params.h"
#include "structs.h"

/* GPU.h:9-27 */
void gridIndexingGPU(unsigned int* DBSIZE, uint64_t totalCells, DTYPE* database, DTYPE** dev_database,
                     DTYPE* epsilon, DTYPE** dev_epsilon, DTYPE* minArr, DTYPE** dev_minArr, struct grid** index,
                     struct grid** dev_index, unsigned int* indexLookupArr, unsigned int** dev_indexLookupArr,
                     struct gridCellLookup** gridCellLookupArr, struct gridCellLookup** dev_gridCellLookupArr,
                     unsigned int* nNonEmptyCells, unsigned int** dev_nNonEmptyCells, unsigned int* nCells,
                     unsigned int** dev_nCells);

/* SortByWorkload.h:7-30 */
void sortByWorkLoad(unsigned int searchMode, unsigned int* DBSIZE, float* staticPartition, uint64_t* totalCandidates,
                    struct schedulingCell** sortedDatabaseTmp, DTYPE* epsilon, DTYPE** dev_epsilon, DTYPE* database,
                    DTYPE** dev_database, struct grid* index, struct grid** dev_index, unsigned int* indexLookupArr,
                    unsigned int** dev_indexLookupArr, struct gridCellLookup* gridCellLookupArr,
                    struct gridCellLookup** dev_gridCellLookupArr, DTYPE* minArr, DTYPE** dev_minArr,
                    unsigned int* nCells, unsigned int** dev_nCells, unsigned int* nNonEmptyCells,
                    unsigned int** dev_nNonEmptyCells, unsigned int** originPointIndex,
                    unsigned int** dev_originPointIndex);

/* GPU.h:29-54 */
void distanceTableNDGridBatches(int searchMode, float staticPartition, unsigned int* DBSIZE, DTYPE* epsilon,
                                DTYPE* dev_epsilon, DTYPE* database, DTYPE* dev_database, struct grid* index,
                                struct grid* dev_index, unsigned int* indexLookupArr, unsigned int* dev_indexLookupArr,
                                struct gridCellLookup* gridCellLookupArr, struct gridCellLookup* dev_gridCellLookupArr,
                                DTYPE* minArr, DTYPE* dev_minArr, unsigned int* nCells, unsigned int* dev_nCells,
                                unsigned int* nNonEmptyCells, unsigned int* dev_nNonEmptyCells,
                                unsigned int* originPointIndex, unsigned int* dev_originPointIndex,
                                struct neighborTableLookup* neighborTable,
                                std::vector<struct neighborDataPtrs>* pointersToNeighbors, uint64_t* totalNeighbors,
                                unsigned int* nbQueriesGPU);

/* GPU.h:90-95 (host helper; this version never reads past pointIDKey[cnt - 1]) */
void constructNeighborTableKeyValueWithPtrs(int* pointIDKey, int* pointInDistValue,
                                            struct neighborTableLookup* neighborTable, int* pointersToNeighbors,
                                            unsigned int* cnt);

/* GPU.h:97 */
void warmUpGPU();

/* main.h:9-16, implemented in hegjoin_b200/compat/hegjoin_import.cpp (link it in
 * place of import_dataset.cpp): the same text and raw-binary formats and the same
 * values, parsed by the library's parallel importer (hj_import_text). */
void importNDDataset(std::vector<std::vector<DTYPE> >* dataPoints, char* fname);
void importNDDatasetBinary(std::vector<std::vector<DTYPE> >* dataPoints, char* fname);

#endif /* HEGJOIN_COMPAT_H */
