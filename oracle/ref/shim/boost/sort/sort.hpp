// Build-only stand-in for Boost.Sort (not installed in this image): the
// reference's Super-EGO path calls boost::sort::sample_sort(first, last, comp,
// threads) once to EGO-sort its points (main.cu:306).  The GNU parallel-mode
// sort gives the same ordering contract (a sort by `comp`) on `threads` cores.
#pragma once
#include <omp.h>
#include <parallel/algorithm>

namespace boost {
namespace sort {
template <class It, class Cmp>
void sample_sort(It first, It last, Cmp comp, unsigned threads) {
    int old = omp_get_max_threads();
    omp_set_num_threads((int)(threads ? threads : 1));
    __gnu_parallel::sort(first, last, comp);
    omp_set_num_threads(old);
}
}  // namespace sort
}  // namespace boost
