// ego_driver.cu -- TEST AND BENCHMARK INFRASTRUCTURE: times the reference's own
// CPU join (Super-EGO, the join of algorithm 3) on a bounded query sample.
//
// It prepares the points exactly as main.cu does for the Super-EGO thread --
// Util::eps / eps2 (main.cu:83-84), the Point array (main.cu:104-118),
// Util::reorderDim (main.cu:298), the EGO sort with egoSortFunction
// (main.cu:306) and the id -> position mapping (main.cu:313-318) -- and then
// calls the reference's Util::egoJoinV2 for each sampled query the way
// Util::multiThreadJoinWorkQueue does (MultiThreadJoin.cpp:116-203), on all
// host cores.  Only the egoJoinV2 calls are timed, like main.cu's egoTime.
//
// usage: ego_driver <dataset.bin> <eps> <target_seconds>
// prints: HJEGO {"queries": m, "pairs": p, "seconds": t, "threads": c, ...}
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <omp.h>

#include <boost/sort/sort.hpp>

#include "params.h"
#include "structs.h"
#include "Point.hpp"
#include "Util.hpp"

bool egoSortFunction(Point const& p1, Point const& p2);   // main.cu:31

static double run_sample(pPoint A, int n, const std::vector<unsigned>& egoMapping, const std::vector<unsigned>& qids,
                         uint64_t* pairs_out) {
    std::vector<uint64_t> nbCandidatesArray(n, 0);
    uint64_t pairs = 0;
    double t0 = omp_get_wtime();
#pragma omp parallel reduction(+ : pairs)
    {
        uint64_t nbCand = 0;
        std::vector<int> result;
#pragma omp for schedule(dynamic, 1)
        for (long s = 0; s < (long)qids.size(); ++s) {
            unsigned index = egoMapping[qids[s]];
            result.clear();
            Util::egoJoinV2(A, 0, n - 1, A, index, index, 0, &nbCand, &result, nbCandidatesArray.data());
            pairs += result.size();
        }
    }
    *pairs_out = pairs;
    return omp_get_wtime() - t0;
}

int main(int argc, char** argv) {
    if (argc != 4) { fprintf(stderr, "usage: %s dataset.bin eps target_seconds\n", argv[0]); return 1; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) { perror(argv[1]); return 1; }
    uint32_t hdr[3];
    if (fread(hdr, 4, 3, f) != 3 || hdr[1] != GPUNUMDIM || hdr[2] != sizeof(REAL)) { fprintf(stderr, "bad dataset\n"); return 1; }
    const int n = (int)hdr[0];
    std::vector<REAL> flat((size_t)n * GPUNUMDIM);
    if (fread(flat.data(), sizeof(REAL), flat.size(), f) != flat.size()) { fprintf(stderr, "short read\n"); return 1; }
    fclose(f);
    const double target = atof(argv[3]);
    DTYPE epsilon = atof(argv[2]);
    Util::eps = epsilon;
    Util::eps2 = epsilon * epsilon;

    pPoint A = new Point[n + 1];
    for (int i = 0; i < n; ++i) {
        A[i].id = i;
        for (int j = 0; j < GPUNUMDIM; ++j) A[i].x[j] = flat[(size_t)i * GPUNUMDIM + j];
    }
    double t0 = omp_get_wtime();
    Util::reorderDim(A, n, A, n);
    double t1 = omp_get_wtime();
    boost::sort::sample_sort(A, A + n, egoSortFunction, CPU_THREADS);
    double t2 = omp_get_wtime();
    std::vector<unsigned> egoMapping(n);
    for (int i = 0; i < n; ++i) egoMapping[A[i].id] = i;

    // size the sample on 64 evenly spaced queries, then run ~target seconds
    auto spaced = [&](int m) {
        std::vector<unsigned> q(m);
        for (int s = 0; s < m; ++s) q[s] = (unsigned)((int64_t)s * (n - 1) / std::max(1, m - 1));
        return q;
    };
    uint64_t pairs = 0;
    double tp = run_sample(A, n, egoMapping, spaced(64), &pairs);
    int m = (int)std::min<double>(n, std::max(64.0, 64.0 * target / std::max(tp, 1e-3)));
    double t = run_sample(A, n, egoMapping, spaced(m), &pairs);
    printf("HJEGO {\"queries\": %d, \"pairs\": %llu, \"seconds\": %.6f, \"threads\": %d, \"n\": %d, "
           "\"reorder_s\": %.6f, \"sort_s\": %.6f}\n",
           m, (unsigned long long)pairs, t, omp_get_max_threads(), n, t1 - t0, t2 - t1);
    delete[] A;
    return 0;
}
