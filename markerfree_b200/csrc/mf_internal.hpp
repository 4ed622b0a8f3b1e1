// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/markerfree.h"

namespace mf {

// Reference constants (Markerfree/src/method/Util.h:33, CalcReproj.cu:12).
constexpr double kD2R = 3.14159265358979323846 / 180.0;
constexpr float kBpD2R = 0.01745f;
constexpr float kSentinel = -1e30f;

// ---- error reporting ------------------------------------------------------
int set_error(int code, const char* fmt, ...);
#define MF_CHECK_CUDA(call)                                                          \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return mf::set_error(MF_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                           cudaGetErrorString(e_));                                  \
  } while (0)
#define MF_CHECK_CUFFT(call)                                                         \
  do {                                                                               \
    cufftResult r_ = (call);                                                         \
    if (r_ != CUFFT_SUCCESS)                                                         \
      return mf::set_error(MF_ERR_CUFFT, "%s:%d %s: cufft error %d", __FILE__,       \
                           __LINE__, #call, (int)r_);                                \
  } while (0)
#define MF_TRY(expr)          \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != MF_OK) return rc_; \
  } while (0)
#define MF_LAUNCHED(ctx) ((ctx)->launches++)

// Correctly rounded float trig: the reference evaluates cosf/sinf (device) or
// (float)cos(double) (host); both sides of every parity check here use this.
inline float cos_f(float x) { return (float)std::cos((double)x); }
inline float sin_f(float x) { return (float)std::sin((double)x); }

// ---- device buffer --------------------------------------------------------
// Buffers are allocated stream-ordered (cudaMallocAsync) on the stream of the
// context that the current API call runs on, from the device's default pool,
// whose release threshold the context raises so that freed memory is reused by
// the next series instead of going back to the driver.
void set_alloc_stream(cudaStream_t s);
// While set, buffers are released with a synchronous cudaFree (used when the
// owning stream may already be gone).
void set_sync_free(bool on);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int alloc(size_t n);  // keeps the existing allocation when large enough
  void release();
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// cuFFT plan wrapper; plans are created on first use and bound to a stream.
struct FftPlan {
  cufftHandle h = 0;
  bool valid = false;
  std::vector<long long> key;
  ~FftPlan();
  void release();
};

struct Context {
  int gpu = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;  // library kernel launches queued (for reporting)
  int sm_count = 148;
  bool profiling = false;
  double stage[6] = {0, 0, 0, 0, 0, 0};  // see mf_context_stage_times
};

// ---- per-held-out-tilt banded re-projection operator ----------------------
// For held-out tilt ip the back-projection of neighbours [i0, i1] into the slab
// followed by the ray sum is, for every image row alike, a linear map from the
// neighbour rows to the re-projected row.  Columns are grouped in tiles of
// kOpTileX; for tile t and neighbour k the map touches input columns
// [lo, hi]; those rows are stacked into a dense (R_t x kOpTileX) block.
constexpr int kOpTileX = 64;
constexpr int kOpChunk = 16;  // R_t is padded to a multiple of this

struct OpTile {
  int row0;  // first row of this tile in the concatenated coefficient matrix
  int rows;  // padded number of rows
};

// One held-out tilt's operator inside a ReprojOpSet (device pointers).
struct ReprojOpView {
  int ip = -1, i0 = -1, nk = 0, xb = 0, yb = 0, ntiles = 0, total_rows = 0;
  const float* coef = nullptr;      // float [rows][kOpTileX], rows indexed by OpTile::row0
  const int2* rowmap = nullptr;     // int2 [rows] = (absolute tilt index, column)
  const OpTile* tiles = nullptr;    // OpTile [ntiles] of this tilt
  const int* colvalid = nullptr;    // int [xb]: ray validity (count >= 0.8 L)
};

// Operators of many held-out tilts in one set of allocations.
struct ReprojOpSet {
  DevBuf coef, rowmap, tiles, colvalid;
  std::vector<ReprojOpView> ops;
  double bytes = 0;  // compulsory bytes of one apply of every operator
  double fma = 0;    // multiply-adds of one apply of every operator
};

// ---- kernels (launch wrappers; all ordered on `st`) -------------------------
// Resample (rotate+shift, nearest) + bin one or more tilts of `stack`
// (nz x ny x nx) using per-tilt device parameters; tilts listed in d_tilts.
// Output tilt j (j-th entry of d_tilts) goes to out + j*out_tilt_stride with row
// stride out_row_stride.
int launch_correct_bin(Context* c, const float* stack, int nx, int ny, const int* d_tilts,
                       int ntilts, const float* d_sx, const float* d_sy, const float* d_rot,
                       int only_shift, int bin, int random_fill, float* out, int out_row_stride,
                       size_t out_tilt_stride, cudaStream_t st);
// Same for a single image with scalar parameters.
int launch_correct_one(Context* c, const float* img, int nx, int ny, float sx, float sy,
                       float axis_deg, int only_shift, int bin, int random_fill, float* out,
                       int out_row_stride, cudaStream_t st);
// Multiply rows of R2C spectra by the R-weight filter (CorrStack.cu:431-446).
int launch_rweight(Context* c, cufftComplex* spec, int cmp, int rows, cudaStream_t st);

// Exact per-sample gather re-projection (CalcReproj.cu:17-124), all rows.
// If d_rowflags != nullptr only row tiles (kApplyTileY rows) whose flag is set
// are processed.
int launch_reproject_exact(Context* c, const float* corr, int xb, int yb, size_t pix,
                           const float* d_bp /*[nk][3] w,c,s*/, int i0, int nk, float fcos,
                           float fsin, int ray_len, int thick, const int* d_rowflags,
                           float* out, cudaStream_t st);
constexpr int kApplyTileY = 128;  // rows per apply tile (and per sentinel flag)
int launch_reproject_apply(Context* c, const ReprojOpView& op, const float* corr, size_t pix,
                           int* d_rowflags, float* out, cudaStream_t st);

// Host-side geometry shared by the operator builder and the exact kernel.
struct ReprojGeom {
  int ip, i0, i1, nk, xb, yb, thick, ray_len;
  float fcos, fsin;
  std::vector<float> bp;  // nk x (w, c, s)
};
void reproj_geometry(const float* angles, int ip, int i0, int i1, int xb, int yb, int thick,
                     ReprojGeom* g);
// Builds the operators of all geometries (same xb, yb) with two launches.
int build_reproj_ops(Context* c, const std::vector<ReprojGeom>& geoms, ReprojOpSet* set,
                     cudaStream_t st);

void find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                     int nproj, int* range);
int frame_idx_from_tilt(int nz, const float* a, float tilt);
int find_ref_index(int nz, const float* a, int z);

}  // namespace mf
