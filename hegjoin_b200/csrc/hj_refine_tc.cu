// hj_refine_tc.cu -- tensor-core distance filter (placeholder until the tcgen05 kernel lands).
#include "hj_internal.h"

namespace hj {
bool tc_supported(const hj_index*, int) { return false; }
uint32_t tc_query_block() { return 512; }
double tc_delta(const hj_index*) { return 0.0; }
hj_status tc_prepare(hj_index*, int, cudaStream_t) {
    set_error("tensor-core filter not built");
    return HJ_ERR_UNSUPPORTED;
}
hj_status launch_refine_tc(const hj_index*, const HjBlock*, uint32_t, unsigned int*, const PairSink&, uint32_t,
                           unsigned long long*, double, unsigned long long*, cudaStream_t) {
    set_error("tensor-core filter not built");
    return HJ_ERR_UNSUPPORTED;
}
}  // namespace hj
