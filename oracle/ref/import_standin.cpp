// Stand-in for import_dataset.cpp in float builds of the reference, whose own
// file does not compile when DTYPE is float (its unused binary importer,
// import_dataset.cpp:82, assigns a double* to a DTYPE*).  importNDDataset here
// parses the same comma/newline text the same way (getline on ',' then
// stringstream >> DTYPE per token, import_dataset.cpp:10-40), so the reference
// CLI reads identical values.
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <cstdio>

#include "params.h"

void importNDDataset(std::vector<std::vector<DTYPE> >* dataPoints, char* fname) {
    std::vector<DTYPE> all;
    std::ifstream in(fname);
    for (std::string f; std::getline(in, f, ',');) {
        DTYPE v;
        std::stringstream ss(f);
        while (ss >> v) {
            all.push_back(v);
            if (ss.peek() == ',') ss.ignore();
        }
    }
    const unsigned total = (unsigned)all.size() / GPUNUMDIM;
    for (unsigned i = 0; i < total; ++i)
        dataPoints->push_back(std::vector<DTYPE>(all.begin() + (size_t)i * GPUNUMDIM,
                                                 all.begin() + (size_t)(i + 1) * GPUNUMDIM));
    printf("Data import: Total data points: %u\n", total);
}
