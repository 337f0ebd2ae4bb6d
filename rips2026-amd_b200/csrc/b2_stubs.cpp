// Entry points whose kernels are not built yet report B2_NOT_SUPPORTED.
#include "../../include/b200sssp.h"

extern "C" b2_status b2_sssp_adds(b2_graph, uint32_t, void*, int32_t*, const b2_sssp_opts*, b2_stream,
                                  b2_stats*) { return B2_NOT_SUPPORTED; }
extern "C" b2_status b2_sssp_bf_dense(const float*, int32_t, uint32_t, float*, const b2_sssp_opts*,
                                      b2_stream, b2_stats*) { return B2_NOT_SUPPORTED; }
extern "C" b2_status b2_minplus_spgemm_f32(const b2_csr*, const b2_csr*, int64_t**, int32_t**, float**,
                                           int64_t*, b2_stream) { return B2_NOT_SUPPORTED; }
extern "C" b2_status b2_minplus_spgemm_i32(const b2_csr*, const b2_csr*, int64_t**, int32_t**, int32_t**,
                                           int64_t*, b2_stream) { return B2_NOT_SUPPORTED; }
