// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <array>
#include <cmath>
#include <cstdio>
#include <functional>
#include <mutex>
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
// The lock every cuFFT call and stream capture of the process holds (mf_series.cu).
std::recursive_mutex& fft_mutex();
#define MF_CHECK_CUDA(call)                                                          \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return mf::set_error(MF_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                           cudaGetErrorString(e_));                                  \
  } while (0)
#define MF_CHECK_CUFFT(call)                                                         \
  do {                                                                               \
    std::lock_guard<std::recursive_mutex> fft_lk_(mf::fft_mutex());                  \
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
// Device allocations number first .. first+count-1 from now on fail (test hook).
void fail_device_allocations(long long first, long long count);
// The stream DevBuf::release frees on in this thread (null: each buffer's own).
void set_free_stream(cudaStream_t s);

// MRC helpers shared by the file entry points (mf_io.cpp): the float32 output
// header from the middle slice, and an input stack opened at its first data byte.
void mrc_float_header(const float* mid, int nx, int ny, int nz, void* out1024);
int mrc_open_stack(const char* path, FILE** fp, int* nx, int* ny, int* nz, int* mode);

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

// Page-locked host slots for results that kernels deliver to the host: a copy into
// pageable memory would make the host wait for the stream at the copy, so the
// stages that queue work for many series before waiting once copy their results
// here instead.  Slot i grows (cudaHostAlloc) the first time it is asked for more
// bytes and is kept for the context's lifetime.
struct PinnedSlots {
  std::vector<std::pair<void*, size_t>> slot;
  void* get(int i, size_t bytes);  // nullptr (error set) when the allocation fails
  PinnedSlots() = default;
  PinnedSlots(const PinnedSlots&) = delete;
  PinnedSlots& operator=(const PinnedSlots&) = delete;
  ~PinnedSlots();
};

// cuFFT plan wrapper; plans are created on first use and bound to a stream.
struct FftPlan {
  cufftHandle h = 0;
  bool valid = false;
  std::vector<long long> key;
  ~FftPlan();
  void release();
};

// Stages of Context::breakdown: series creation (upload, pre-processing, the
// column-major copy), coarse alignment (stretch correlations, offset search),
// tilt-axis searches, projection-matching set-up, projection-matching passes,
// aligned-stack output; then the Radon kernel of the tilt-axis searches on its
// own: its time, launches, samples taken and compulsory bytes.
enum StageSlot { kStagePrep, kStageCoarse, kStageAxis, kStageSetup, kStagePass, kStageFinal,
                 kStageRadonMs, kStageRadonLaunches, kStageRadonSamples, kStageRadonBytes,
                 kStages };

struct Context {
  int gpu = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;  // library kernel launches queued (for reporting)
  int sm_count = 148;
  bool profiling = false;
  int tc_rows = 0;  // tensor-core tile rows (64/128/256); 0 = chosen per shape
  // tile rows the autotuner chose, per (xb, yb, jobs, precision)
  std::vector<std::array<int, 5>> tc_tuned;
  // median ms per launch the autotuner measured for 256/128/64 rows, per entry of tc_tuned
  std::vector<std::array<float, 3>> tc_tuned_ms;
  PinnedSlots pinned;  // host result slots of the queued stages
  double stage[6] = {0, 0, 0, 0, 0, 0};  // see mf_context_stage_times
  double breakdown[kStages] = {};        // ms per stage, see mf_context_stage_breakdown
};

// Wall time on the context's stream of one stage of an alignment, accumulated in
// Context::breakdown when profiling is on (events on both sides, then a wait).
class StageTimer {
 public:
  StageTimer(Context* c, int slot) : c_(c), slot_(slot) {
    if (!c->profiling) return;
    if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    on_ = cudaEventRecord(a_, c->stream) == cudaSuccess;
  }
  ~StageTimer() {
    if (on_ && cudaEventRecord(b_, c_->stream) == cudaSuccess &&
        cudaEventSynchronize(b_) == cudaSuccess) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, a_, b_) == cudaSuccess) c_->breakdown[slot_] += ms;
    }
    if (a_) cudaEventDestroy(a_);
    if (b_) cudaEventDestroy(b_);
    cudaGetLastError();
  }
  StageTimer(const StageTimer&) = delete;
  StageTimer& operator=(const StageTimer&) = delete;

 private:
  Context* c_;
  int slot_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
  bool on_ = false;
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

// ---- tensor-core (tcgen05) form of the same operator ------------------------
// Used by the FP16/BF16 precision modes: operator coefficients and neighbour rows
// in 16 bits, products accumulated in FP32 in tensor memory.  Output columns are
// grouped in x-tiles of kTcM = 128 (the MMA's M).  For x-tile t and neighbour k
// the touched bins [lo, hi] become a segment starting at b0 = lo rounded down to
// a multiple of 8 (a TMA box must start on a 16-byte boundary) and covering
// nch chunks of kTcK = 64 bins (one 128-byte swizzle row of 16-bit values).
// Chunk c of the operator is a 128 x 64 block stored K-major: the 64
// coefficients of output column m are contiguous, at op16 + (c*128 + m)*64.
// Coefficients are stored multiplied by kTcScale (a power of two that keeps them
// inside the FP16 normal range); the epilogue divides it out exactly.
constexpr int kTcM = 128;
constexpr int kTcK = 64;
constexpr float kTcScale = 64.0f;
struct TcSeg {
  int tilt;    // absolute tilt index of the neighbour
  int b0;      // first bin of the segment (multiple of 8)
  int nch;     // chunks of kTcK bins
  int chunk0;  // first chunk of the segment in the operator
};
struct TcXTile {
  int seg0;  // first segment of this x-tile in the segment table
  int nseg;
  int nch;   // chunks over all segments
  int pad;
};
// Opaque storage for a CUtensorMap (the driver type is 64-byte aligned, 128 B).
struct alignas(64) TmaDesc {
  unsigned char b[128];
};
struct TcOpView {
  int ip = -1, i0 = 0, nk = 0, xb = 0, yb = 0, ntx = 0, nchunks = 0;
  const TcXTile* xt = nullptr;  // [ntx] (segment indices are global)
  const TcSeg* segs = nullptr;  // the set's whole segment table
  const int* colvalid = nullptr;
};
struct TcOpSet {
  DevBuf op16, xt, segs, colvalid;
  std::vector<TcOpView> ops;
  int total_chunks = 0;
  int nsegs = 0, nxt = 0;  // entries of segs and xt
  int half_kind = 0;  // MF_PREC_BF16 or MF_PREC_FP16
  TmaDesc opmap;      // 2-D tensor map over op16, box 64 x 128
  double bytes = 0;   // compulsory bytes of one apply of every operator
  double fma = 0;     // multiply-adds issued to the tensor cores
};

// ---- kernels (launch wrappers; all ordered on `st`) -------------------------
// Resample (rotate+shift, nearest) + bin one or more tilts of `stack`
// (nz x ny x nx) using per-tilt device parameters; tilts listed in d_tilts.
// Output tilt j (j-th entry of d_tilts) goes to out + j*out_tilt_stride with row
// stride out_row_stride.
// stack_t: the stack's column-major copy (nz x nx x ny), or null; read for tilts
// whose axis makes output rows run along source columns.
int launch_correct_bin(Context* c, const float* stack, const float* stack_t, int nx, int ny,
                       const int* d_tilts, int ntilts, const float* d_sx, const float* d_sy,
                       const float* d_rot, int only_shift, int bin, int random_fill, float* out,
                       int out_row_stride, size_t out_tilt_stride, cudaStream_t st);
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
// The (w, cos, sin) table of every geometry evaluated on the device with CUDA's
// cosf/sinf, as the reference's back-projection kernel does, written back into
// geoms[i].bp (the host values of reproj_geometry are correctly rounded).
constexpr int kMaxBpNeighbours = 256;
int fill_bp_device(Context* c, const float* angles, std::vector<ReprojGeom>* geoms,
                   cudaStream_t st);
// The same table for one held-out tilt straight into device memory.
int bp_table_device(Context* c, const float* angles, int ip, int i0, int nk, float* d_out,
                    cudaStream_t st);
// Builds the operators of all geometries (same xb, yb) with two launches.
int build_reproj_ops(Context* c, const std::vector<ReprojGeom>& geoms, ReprojOpSet* set,
                     cudaStream_t st);

// Tensor-core operators of all geometries (same xb, yb) in `half_kind` precision.
int build_reproj_tc_ops(Context* c, const std::vector<ReprojGeom>& geoms, int half_kind,
                        TcOpSet* set, cudaStream_t st);
// The same two builders for geometries of any image sizes: one set per size, then
// concatenated into `set` (ops in the order of `geoms`).
int build_reproj_ops_any(Context* c, const std::vector<ReprojGeom>& geoms, ReprojOpSet* set,
                         cudaStream_t st);
int build_reproj_tc_ops_any(Context* c, const std::vector<ReprojGeom>& geoms, int half_kind,
                            TcOpSet* set, cudaStream_t st);
// Encodes set->opmap over set->op16 (called by build_reproj_tc_ops).
int tc_op_map(TcOpSet* set);
// 3-D tensor map over a 16-bit copy of the corrected stack (nz x yb rows of xb
// values with row pitch `xpitch` elements), box 64 bins x nb rows.
int tc_image_map(const void* base, int half_kind, int xb, int xpitch, int yb, int nz, int nb,
                 TmaDesc* out);
// Rows per tensor-core tile (the MMA's N) for an image shape: the context's
// override if set, else the widest of 256/128/64 that still gives most SMs a tile.
int tc_pick_rows(const Context* c, int xb, int yb);
// Autotuner of the tile rows: times `launch(nb)` (one re-projection step with
// tiles of nb rows, queued on st) for nb = 64, 128, 256 -- one untimed launch,
// then the median of five timed ones -- keeps the fastest for the shape (xb, yb,
// jobs, precision) in the context and returns it in *nb_out.  The kernel's
// pipeline error word d_err is cleared before each variant and read after it: a
// variant whose bounded waits gave up fails the call with MF_ERR_CUDA instead of
// looking fast.  A shape seen before, or tile rows fixed with
// mf_context_set_tc_rows, is not timed again.
int tc_autotune_rows(Context* c, int xb, int yb, int jobs, int prec,
                     const std::function<int(int)>& launch, int* d_err, int* nb_out,
                     cudaStream_t st);
// Sets the kernel attributes of the tile-rows variant `nb` on the current device
// (done outside any stream capture).
int tc_prepare(Context* c, int nb);
// out (yb x xb) = tensor-core apply of one operator to the 16-bit stack behind
// `imgmap`; columns without a valid ray get -1e30.  *d_err becomes non-zero if a
// pipeline wait gave up (the kernel then returns without finishing).
int launch_reproject_tc(Context* c, const TcOpSet& set, const TcOpView& op, const TmaDesc& imgmap,
                        int nb, int* d_err, float* out, cudaStream_t st);
// FP32 corrected images -> 16-bit copy (row pitch xpitch) for tilts d_tilts[0..n)
// (or tilts tilt0..tilt0+n-1 when d_tilts is null).  tflags[tilt * ytiles + t]
// is set when 128-row tile t of the tilt holds a value the 16-bit path cannot
// carry (a -1e30 sentinel, a NaN, or a magnitude beyond the FP16 range).
int launch_to_half(Context* c, const float* src, int xb, int yb, const int* d_tilts, int tilt0,
                   int n, int half_kind, void* dst, int xpitch, int* tflags, cudaStream_t st);
// Exact re-projection of the 128-row tiles of `out` whose neighbour tilts
// [i0, i0+nk) have a tflags entry set (the fallback after the tensor-core apply).
int launch_reproject_exact_flagged(Context* c, const float* corr, int xb, int yb, size_t pix,
                                   const float* d_bp, int i0, int nk, float fcos, float fsin,
                                   int ray_len, int thick, const int* tflags, float* out,
                                   cudaStream_t st);

// ---- multi-series (group) execution ------------------------------------------
// A group runs the projection-matching pass of up to kMaxGroup series in
// lockstep: every stage is one launch over all series of the group (the k-th
// held-out tilt of every series together).  Series may differ in every size --
// image, tilt count, slab thickness, matching binning -- so each kernel reads the
// geometry and the work buffers of its series from the series' GroupSeriesDev
// record and the grid covers the largest series; blocks beyond a smaller series'
// extent return at once.  A series with fewer held-out tilts has no work in the
// last steps (its GroupStepDev::ip is -1 there), and a per-series `active` flag
// skips series that have already left the current ProjAlignOnce loop.  Every
// series' arithmetic and its order are those of the series aligned alone.
constexpr int kMaxGroup = 32;
constexpr int kFlagParts = 8;  // column parts of a 16-bit copy's per-tile flags

struct GroupSeriesDev {
  const float* stack;    // pre-processed stack (nz x ny x nx)
  const float* stack_t;  // the same, column-major per tilt (nz x nx x ny)
  float* sx;
  float* sy;
  // FP16/BF16 modes: the FP64 accumulators of the shifts (sx/sy hold their float
  // values); null in FP32 mode, where shifts accumulate in float as in the reference
  double* sx64;
  double* sy64;
  const float* rot;
  const float* angles;
  float* z0;
  float* err;    // nz: |shift| of the last measurement per tilt
  float* meas;   // 2 * nz: shift measured in the last pass (un-binned px, before rotation)
  float* corr;   // corrected stack of this series (nz x yb x xb)
  const int* order;  // outward processing order (n entries)
  int zt, n;         // zero-tilt index; held-out tilts per pass (nz - 1)
  // shape (ProjAlign::Setsize, ProjAlign.cpp:48-125; CorrStack.cu:65-100)
  int nx, ny, nz, bin;          // raw image, tilts, matching binning
  int out_x, binx, biny;        // resampling grid before binning, bin factors
  int xb, yb, pad, cmp;         // binned image, padded FFT row (floats), spectrum width
  int ytiles, xpitch;           // 128-row tiles; 16-bit row pitch
  size_t bpix, ppix;            // xb * yb, pad * yb
  // work buffers of the pass
  float* scratch;      // nz x yb x pad: rows of the batched R-weight FFT
  float* reproj;       // yb x xb: re-projection of the step's held-out tilt
  float* cc;           // 2 x yb x pad: the normalised pair, then spectrum / correlation
  float* recorr;       // yb x pad: re-corrected held-out tilt before its R-weight
  const float* mask;   // yb x xb round-edge factors of the correlation mask
  double2* mpart;      // 2 x moment_parts(yb) moment partials
  float2* stats;       // 2: (mean, std) of the pair
  float2* ppart;       // kPeakParts peak partials
  void* corr16;        // FP16/BF16: nz x yb x xpitch 16-bit copy of corr
  int* tflags;         // nz x ytiles x kFlagParts flags: tiles the operator cannot carry
};
struct GroupStepDev {  // the held-out tilt of one series at one step of the pass
  int ip, i0, nk, ray_len, thick, bp_off;  // ip < 0: the series has no tilt at this step
  float fcos, fsin;
};
struct GroupCorrArgs {
  const GroupSeriesDev* ser;
  const GroupStepDev* steps;  // null: all tilts of every series (job = b * nz_max + tilt)
  const int* active;          // null: all series
  int nz_max, random_fill;
};
// resample + bin (k_correct_bin) for a group; all tilts (steps == null) into each
// series' scratch rows, or each series' held-out tilt of a step into its recorr
int launch_correct_group(Context* c, const GroupCorrArgs& a, int nseries, int xb_max, int yb_max,
                         cudaStream_t st);
// R-weight (k_rweight) of every series' scratch rows (steps == null) or of its
// re-corrected tilt at a step
int launch_rweight_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                         const int* active, int nseries, int cmp_max, int rows_max,
                         cudaStream_t st);
// FP32 -> 16-bit copy (launch_to_half) of every tilt (steps == null) or of each
// series' held-out tilt of a step
int launch_to_half_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                         const int* active, int nseries, int nz_max, int ytiles_max,
                         int half_kind, cudaStream_t st);
// exact re-projection of the flagged 128-row tiles of every active series at one
// step into its reproj buffer; flags: the series' tflags when tc (16-bit copy or
// FP32 sentinel flags), else rowflags of the step (rowflags[b * ytiles_max + tile])
int launch_reproject_exact_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                                 const int* active, int nseries, int xb_max, int ytiles_max,
                                 const float* d_bp, bool tc, const int* rowflags,
                                 cudaStream_t st);
// FP32 groups: per-(tilt, 128-row tile, column part) sentinel flags of the
// corrected stacks (the tflags layout of the 16-bit copies), for all tilts of
// every series (steps == null) or each series' held-out tilt of a step
// Per-(tilt, 128-row tile, column part) sentinel flags of one series' FP32
// corrected stack (xb even): every tilt (d_tilts null) or the listed ones.
int launch_flag_tiles(Context* c, const float* corr, int xb, int yb, const int* d_tilts,
                      int ntilts, int* tflags, cudaStream_t st);
int launch_flag_tiles_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                            const int* active, int nseries, int nz_max, int ytiles_max,
                            cudaStream_t st);
struct ApplyJob {  // one series of a group at one step of the FP32 apply
  const OpTile* tiles;
  const int* colvalid;
  const float* corr;
  float* out;
  int* rowflags;
  int xb, yb, ntiles;  // ntiles 0: no held-out tilt at this step
};
// Sets the group apply's shared-memory attribute for the device (once; call it
// outside stream capture).
int prepare_apply_group(Context* c);
int launch_reproject_apply_group(Context* c, const ReprojOpSet& set, const ApplyJob* d_jobs,
                                 const int* active, int njobs, int ntiles_max, int yb_max,
                                 cudaStream_t st);
struct TcJob {
  const TcXTile* xt;
  const int* colvalid;
  float* out;
  int series;        // index into `active`
  int map;           // image tensor map of this series
  int xb, yb, ntx;   // output size and 128-column tiles
  int tile0;         // first tile of this job in the launch (set when launched)
};
// Tensor-core apply for a list of jobs (series of any shapes); maps[j] is the
// 16-bit image map of job j's series.
int launch_reproject_tc_group(Context* c, const TcOpSet& set, const TcJob* jobs, int njobs,
                              const int* active, const TmaDesc* maps, int nmaps, int nb,
                              int* d_err, cudaStream_t st);

void find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                     int nproj, int* range);
int frame_idx_from_tilt(int nz, const float* a, float tilt);
int find_ref_index(int nz, const float* a, int z);

}  // namespace mf
