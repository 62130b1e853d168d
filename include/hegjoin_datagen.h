/* hegjoin_datagen.h -- seeded synthetic datasets (host library libhj_datagen.so).
 *
 * Test and benchmark inputs, not part of the join: the generator stands in for
 * the reference's dataset generator (datasets/dataset_gen_fixed_len_expo_dist.cpp:24-91,
 * i.i.d. Exp(rate=40) per coordinate, values >= 1 redrawn) with a counter-based
 * RNG, so any slice of a dataset can be produced in parallel and reproduced bit
 * for bit.  It is a separate host-only library so that a process timing the
 * reference's CPU path can make the same inputs without loading the GPU
 * library.
 */
#ifndef HEGJOIN_DATAGEN_H
#define HEGJOIN_DATAGEN_H

#include "hegjoin_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* n x d coordinates i.i.d. Exp(rate=40), redrawn into [0, 1) after the cast to
 * the dataset type, from a counter-based generator (seed, stream): the same
 * values hegjoin_b200.workloads.exp40 produces.  Host memory; OpenMP. */
hj_status hj_generate_exp40(uint64_t seed, uint64_t stream, uint64_t n, uint32_t d, int dtype, void* h_out);
/* The skewed workload: the first n - round(frac * n) points from
 * hj_generate_exp40(seed, 0, ...), the rest from n_clusters Gaussian clusters
 * (standard deviation sigma, centres uniform in [0,1)^d), clipped to [0, 1). */
hj_status hj_generate_skewed(uint64_t seed, uint64_t n, uint32_t d, uint32_t n_clusters, double sigma,
                             double frac_clustered, int dtype, void* h_out);

#ifdef __cplusplus
}
#endif

#endif /* HEGJOIN_DATAGEN_H */
