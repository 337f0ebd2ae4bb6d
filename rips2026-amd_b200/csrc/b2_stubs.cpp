// Entry points whose kernels are not built yet report B2_NOT_SUPPORTED.
#include "../../include/b200sssp.h"

extern "C" b2_status b2_sssp_adds(b2_graph, uint32_t, void*, int32_t*, const b2_sssp_opts*, b2_stream,
                                  b2_stats*) { return B2_NOT_SUPPORTED; }
