// C ABI glue: status strings, option defaults, version.
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/b200sssp.h"

extern "C" const char* b2_status_string(b2_status s) {
  switch (s) {
    case B2_SUCCESS: return "success";
    case B2_INVALID_ARGUMENT: return "invalid argument";
    case B2_CUDA_ERROR: return "CUDA error";
    case B2_OUT_OF_MEMORY: return "out of device memory";
    case B2_POOL_EXHAUSTED: return "worklist capacity exhausted";
    case B2_BUCKET_OVERFLOW: return "bucket overflow";
    case B2_DEVICE_ERROR: return "device-side consistency error";
    case B2_TIMEOUT: return "bounded device wait timed out";
    case B2_NOT_SUPPORTED: return "not supported by this build";
    case B2_INVALID_INDEX: return "CSR column index out of range";
    case B2_INVALID_ROWPTR: return "CSR row pointer invalid";
    case B2_INVALID_WEIGHT: return "edge weight not allowed for this method";
    case B2_CANCELLED: return "query cancelled";
  }
  return "unknown status";
}

extern "C" int b2_abi_version(void) { return B2_ABI_VERSION; }

extern "C" void b2_sssp_opts_default(b2_sssp_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->max_iters = -1;
  o->bf_check = B2_BF_CHECKED;
  o->check_interval = 1;
  o->policy = 0;
  o->delta = 0.0;
  o->delta_scale = 16.0;
  o->hub_degree = 256;
  o->fusion_threshold = 0;
  o->pull_fraction = 8.0f;
  o->grid_blocks = 0;
  o->timeout_ms = 20000.0;
  o->collect_reach = 0;
  o->detect_negative_cycle = 0;
  o->light_heavy = 1;
  o->trace = 0;
  o->dense_fraction = 0.0f;
}

extern "C" b2_status b2_device_free(void* p) {
  if (!p) return B2_SUCCESS;
  return cudaFree(p) == cudaSuccess ? B2_SUCCESS : B2_CUDA_ERROR;
}

extern "C" b2_status b2_device_copy(void* dst, const void* src, size_t bytes, b2_stream stream) {
  if (bytes == 0) return B2_SUCCESS;
  if (!dst || !src) return B2_INVALID_ARGUMENT;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  return e == cudaSuccess ? B2_SUCCESS : B2_CUDA_ERROR;
}
