// structs.h for building and testing the compatibility shim without the
// reference tree.  A caller of the shim compiles it against its own structs.h;
// the types here repeat the layouts the shim exchanges with that caller
// (HEGJoin structs.h:35-104): field names, types and order must be identical
// for the two sides to agree on memory layout.
#ifndef STRUCTS_H
#define STRUCTS_H

#include "params.h"

#include <cstdint>
#include <vector>

struct neighborTableLookup {
    int pointID;
    int indexmin;
    int indexmax;   // exclusive
    int* dataPtr;
};

struct neighborDataPtrs {
    int* dataPtr;
    int sizeOfDataArr;
};

struct grid {
    int indexmin;   // inclusive
    int indexmax;   // inclusive
};

struct gridCellLookup {
    unsigned int idx;
    uint64_t gridLinearID;
    bool operator<(const gridCellLookup& other) const { return gridLinearID < other.gridLinearID; }
};

struct schedulingCell {
    int nbPoints;
    int cellId;
};

#endif
