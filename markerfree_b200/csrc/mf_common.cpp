// Error reporting and device buffers.
#include <cstdarg>
#include <cstdio>

#include "mf_internal.hpp"

namespace mf {

static thread_local char g_last_error[1024] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

const char* last_error() { return g_last_error; }

int DevBuf::alloc(size_t n) {
  if (n == 0) n = 16;
  if (p && bytes >= n) return MF_OK;
  release();
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    cudaGetLastError();
    return set_error(MF_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return MF_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

FftPlan::~FftPlan() { release(); }

void FftPlan::release() {
  if (valid) cufftDestroy(h);
  valid = false;
}

}  // namespace mf
