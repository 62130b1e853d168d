// hegjoin_import.cpp -- the reference's dataset importers (main.h:9-16) on top
// of the library's parallel parser.  Compile with the caller's params.h and link
// it in place of import_dataset.cpp.
//
// importNDDataset reads the reference's text format with hj_import_text, which
// follows import_dataset.cpp:10-40 value for value (tokens split at ',',
// `stream >> DTYPE` semantics per token), and fills the caller's vector of
// points the way that function does; it prints the same two lines.
// importNDDatasetBinary reads the reference's raw layout (or the library's
// binary twin) with hj_import_binary.
#include <cstdio>
#include <vector>

#include "hegjoin_b200.h"
#include "hegjoin_compat.h"

namespace {

constexpr int kDtype = sizeof(DTYPE) == sizeof(double) ? HJ_F64 : HJ_F32;

void fill(std::vector<std::vector<DTYPE> >* dataPoints, const DTYPE* vals, uint64_t n) {
    dataPoints->reserve(dataPoints->size() + n);
    for (uint64_t i = 0; i < n; ++i)
        dataPoints->emplace_back(vals + i * GPUNUMDIM, vals + (i + 1) * GPUNUMDIM);
}

}  // namespace

void importNDDataset(std::vector<std::vector<DTYPE> >* dataPoints, char* fname) {
    void* vals = nullptr;
    uint64_t n = 0;
    hj_status s = hj_import_text(fname, GPUNUMDIM, kDtype, &vals, &n);
    if (s != HJ_OK) {
        printf("Data import: Error: %s\n", hj_last_error());
        return;
    }
    printf("Data import: Total size of all data (1-D) vect (number of points * GPUNUMDIM): %zu\n",
           (size_t)(n * GPUNUMDIM));
    printf("Data import: Total data points: %d\n", (int)n);
    fill(dataPoints, static_cast<const DTYPE*>(vals), n);
    hj_host_free(vals);
}

void importNDDatasetBinary(std::vector<std::vector<DTYPE> >* dataPoints, char* fname) {
    void* vals = nullptr;
    uint64_t n = 0;
    hj_status s = hj_import_binary(fname, GPUNUMDIM, kDtype, &vals, &n);
    if (s != HJ_OK) {
        printf("Data import: Error: %s\n", hj_last_error());
        return;
    }
    printf("Data import: Total data points: %d\n", (int)n);
    fill(dataPoints, static_cast<const DTYPE*>(vals), n);
    hj_host_free(vals);
}
