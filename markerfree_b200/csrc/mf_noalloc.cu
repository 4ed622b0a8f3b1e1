// Exact re-projection for callers that must not allocate device memory.
//
// mf_dev_reproject (method 0) needs a small device table per call: for every
// neighbour tilt the back-projection weight and the cosine and sine of its
// angle.  It takes that table from the context's scratch buffers, which grow with
// cudaMalloc.  Some host programs cannot let a library do that: an acquisition
// program that has reserved the GPU's memory for its own frame buffers and
// treats any other allocation as an out-of-memory risk mid-session, or a
// real-time loop in which cudaMalloc/cudaFree, which can synchronise the whole
// device, would stall the detector stream.  The entry point below keeps the table
// in a file-scope __device__ array instead, so it performs no device allocation
// at all (and no host heap allocation either: the table is written by a kernel
// whose arguments carry the angles).
//
// The array is sized for kStaticMaxNeighbours neighbours (3 floats each, 3 KB),
// is held by every GPU that loads this library until the process exits, and is
// shared by all calls: two calls whose kernels overlap on the GPU (for example
// on two streams) race on it.  Each call rewrites all the entries its kernel
// reads, so nothing needs clearing between calls.
#include <mutex>

#include "mf_internal.hpp"

namespace mf {
namespace {

constexpr int kStaticMaxNeighbours = 256;
constexpr int kMaxDevices = 64;

// Per-neighbour (weight, cos, sin) of the back-projection, read by the kernel.
static __device__ __align__(256) float g_neighbour_table[kStaticMaxNeighbours * 3];

std::mutex g_table_mu;
float* g_table_addr[kMaxDevices] = {};

// Device address of g_neighbour_table on the current device.  In host code the
// symbol only names a host-side stand-in, so the address is looked up once per
// device, with that device current.
int table_address(int dev, float** out) {
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(MF_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_table_mu);
  if (!g_table_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_neighbour_table);
    if (e != cudaSuccess || !p)
      return set_error(MF_ERR_CUDA, "cudaGetSymbolAddress of the neighbour table failed: %s",
                       cudaGetErrorString(e));
    g_table_addr[dev] = (float*)p;
  }
  *out = g_table_addr[dev];
  return MF_OK;
}

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" MF_API int mf_dev_reproject_noalloc(void* stream, const float* d_corr, int xb, int yb,
                                               int nz, const float* angles, int iproj,
                                               int istart, int iend, int thickness,
                                               float* d_out) {
  if (!d_corr || !angles || !d_out) return set_error(MF_ERR_ARG, "null argument");
  if (istart < 0 || iend < istart || iend >= nz || iproj < 0 || iproj >= nz || thickness < 2 ||
      xb < 2 || yb < 1)
    return set_error(MF_ERR_ARG, "invalid re-projection range or size");
  const int nk = iend - istart + 1;
  if (nk > kStaticMaxNeighbours)
    return set_error(MF_ERR_ARG,
                     "%d neighbour tilts exceed the allocation-free entry point's maximum of %d",
                     nk, kStaticMaxNeighbours);
  int dev = 0;
  MF_CHECK_CUDA(cudaGetDevice(&dev));
  float* d_table = nullptr;
  MF_TRY(table_address(dev, &d_table));
  // geometry of CalcReproj.cu:43-46 and 301-303: the table is written by a small
  // kernel (its angles travel as kernel arguments), then read by the re-projection
  const float pa = angles[iproj];
  const float fcos = (float)std::cos(kD2R * pa);
  const float fsin = (float)std::sin(kD2R * pa);
  const int ray_len = (int)((float)thickness / fcos + 0.5f);
  cudaStream_t st = (cudaStream_t)stream;
  Context c;  // launch bookkeeping only; owns nothing
  c.gpu = dev;
  MF_TRY(bp_table_device(&c, angles, iproj, istart, nk, d_table, st));
  return launch_reproject_exact(&c, d_corr, xb, yb, (size_t)xb * yb, d_table, istart, nk, fcos,
                                fsin, ray_len, thickness, nullptr, d_out, st);
}
