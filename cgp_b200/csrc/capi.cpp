// Error reporting, option defaults and version of the C ABI.
#include <cstdio>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "cgp_b200_internal.h"

namespace cgp {

namespace {
thread_local std::string g_last_error;
}

cgp_status set_error(cgp_status code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

void clear_error() { g_last_error.clear(); }

}  // namespace cgp

extern "C" {

cgp_status cgp_last_error(char* buf, size_t len) {
  if (buf == nullptr || len == 0) return CGP_ERR_INVALID_ARG;
  std::snprintf(buf, len, "%s", cgp::g_last_error.c_str());
  return CGP_OK;
}

const char* cgp_status_name(cgp_status s) {
  switch (s) {
    case CGP_OK: return "CGP_OK";
    case CGP_ERR_INVALID_ARG: return "CGP_ERR_INVALID_ARG";
    case CGP_ERR_OOM: return "CGP_ERR_OOM";
    case CGP_ERR_CUDA: return "CGP_ERR_CUDA";
    case CGP_ERR_TIMEOUT: return "CGP_ERR_TIMEOUT";
    case CGP_ERR_CANCELLED: return "CGP_ERR_CANCELLED";
    case CGP_ERR_NOT_FOUND: return "CGP_ERR_NOT_FOUND";
    case CGP_ERR_BUSY: return "CGP_ERR_BUSY";
    case CGP_ERR_DEVICE: return "CGP_ERR_DEVICE";
  }
  return "CGP_ERR_UNKNOWN";
}

// Defaults of run_options (puercgp/include/puercgp/core/types.hxx:26-46).
cgp_status cgp_options_init(cgp_options* o) {
  if (o == nullptr) return cgp::set_error(CGP_ERR_INVALID_ARG, "options is NULL");
  std::memset(o, 0, sizeof(*o));
  o->traversal_mode = CGP_MODE_HYBRID;
  o->pull_frontier_ratio = 0.15;
  o->pull_edge_ratio = 0.20;
  o->sssp_pull_edge_ratio = 0.5;
  o->sssp_pull_pair_ratio = 0.5;
  o->use_cuda_graph = 1;
  o->depth_mode = CGP_DEPTH_AUTO;
  return CGP_OK;
}

const char* cgp_version(void) { return "cgp_b200 0.1.0 (sm_100a)"; }

cgp_status cgp_set_device(int32_t device) {
  cgp::clear_error();
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return cgp::set_error(CGP_ERR_CUDA, "no CUDA device");
  }
  if (device < 0 || device >= n) return cgp::set_error(CGP_ERR_INVALID_ARG, "device out of range");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cgp::set_error(CGP_ERR_CUDA, cudaGetErrorString(e));
  return CGP_OK;
}

}  // extern "C"
