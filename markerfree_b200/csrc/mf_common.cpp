// Error reporting and device buffers.
#include <atomic>
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

static thread_local cudaStream_t g_alloc_stream = nullptr;
static thread_local cudaStream_t g_free_stream = nullptr;
static thread_local bool g_sync_free = false;

void set_alloc_stream(cudaStream_t s) { g_alloc_stream = s; }
void set_free_stream(cudaStream_t s) { g_free_stream = s; }
void set_sync_free(bool on) { g_sync_free = on; }

static std::atomic<long long> g_alloc_seq{0}, g_fail_first{0}, g_fail_end{0};

void fail_device_allocations(long long first, long long count) {
  const long long base = g_alloc_seq.load();
  g_fail_first = base + first;
  g_fail_end = count > 0 ? base + first + count : 0;
}

int DevBuf::alloc(size_t n) {
  if (n == 0) n = 16;
  if (p && bytes >= n) return MF_OK;
  release();
  const long long k = g_alloc_seq++;
  if (k < g_fail_end && k >= g_fail_first)
    return set_error(MF_ERR_NOMEM, "device allocation of %zu bytes failed: injected", n);
  st = g_alloc_stream;
  cudaError_t e = st ? cudaMallocAsync(&p, n, st) : cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    st = nullptr;
    cudaGetLastError();
    return set_error(MF_ERR_NOMEM, "device allocation of %zu bytes failed: %s", n,
                     cudaGetErrorString(e));
  }
  bytes = n;
  return MF_OK;
}

void DevBuf::release() {
  if (p) {
    // freed in the order of the stream that last used it: the allocating stream,
    // or the one a caller names (a series that moved to another context)
    cudaStream_t fs = g_free_stream ? g_free_stream : st;
    if (!fs || g_sync_free || cudaFreeAsync(p, fs) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(p);
      cudaGetLastError();
    }
  }
  p = nullptr;
  bytes = 0;
  st = nullptr;
}

void* PinnedSlots::get(int i, size_t bytes) {
  if (i < 0) return nullptr;
  if ((int)slot.size() <= i) slot.resize(i + 1, {nullptr, 0});
  auto& e = slot[i];
  if (e.first && e.second >= bytes) return e.first;
  if (e.first) cudaFreeHost(e.first);
  e = {nullptr, 0};
  size_t n = bytes < 4096 ? 4096 : bytes;
  if (cudaHostAlloc(&e.first, n, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    e.first = nullptr;
    set_error(MF_ERR_NOMEM, "page-locked host allocation of %zu bytes failed", n);
    return nullptr;
  }
  e.second = n;
  return e.first;
}

PinnedSlots::~PinnedSlots() {
  for (auto& e : slot)
    if (e.first) cudaFreeHost(e.first);
  cudaGetLastError();
}

FftPlan::~FftPlan() { release(); }

void FftPlan::release() {
  if (valid) {
    std::lock_guard<std::recursive_mutex> lk(fft_mutex());
    cufftDestroy(h);
  }
  valid = false;
}

}  // namespace mf
