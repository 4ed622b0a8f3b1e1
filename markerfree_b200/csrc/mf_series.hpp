// Device-resident tilt series and the alignment stages that run on it.
#pragma once
#include <map>
#include <memory>

#include "mf_internal.hpp"
#include "mf_xcorr.hpp"

struct mf_context {
  mf::Context c;
  // scratch for the single-kernel entry points
  struct Scratch {
    mf::DevBuf a, b, c, d;
  } scratch;
  std::map<std::vector<long long>, cufftHandle> plans;
  // Side streams that run the per-series cuFFT calls of one group stage side by
  // side (each with plans of its own, so that no work area is shared), forked
  // from and joined back into the context stream with the events below.
  static constexpr int kFftStreams = 4;
  cudaStream_t aux[kFftStreams] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kFftStreams] = {};
  // cuFFT work areas, one per side stream and one (the last) for the context
  // stream, each as large as the largest plan bound to that stream needs: cuFFT
  // would otherwise allocate one per plan, and a context meets many shapes
  void* work[kFftStreams + 1] = {};
  size_t work_bytes[kFftStreams + 1] = {};
  std::vector<void*> retired_work;  // outgrown areas (captured graphs may hold them)
  ~mf_context();
  // Plan cache keyed by (kind, sizes, batch); bound to the context stream, or with
  // a fifth key entry i >= 0 to side stream i.
  int plan(const std::vector<long long>& key, cufftHandle* out);
  int ensure_aux();  // creates the side streams and events on first use
};

namespace mf {

struct ProjAlignState {
  bool ready = false;
  int bin = 1, xb = 0, yb = 0, pad = 0, cmp = 0, thick = 0, nproj = 10;
  int zt = 0;
  float z0 = 0.0f;
  std::vector<int> order;               // outward processing order of held-out tilts
  std::vector<ReprojGeom> geom;         // per entry of `order`
  ReprojOpSet ops;
  DevBuf corr;      // nz x yb x xb corrected (R-weighted) stack
  DevBuf scratch;   // nz x yb x pad rows for the batched R-weight FFT
  DevBuf reproj;    // yb x xb
  DevBuf ccbuf;     // 2 x yb x pad
  DevBuf part;      // reduction partials
  DevBuf stats;     // float2 x 2
  DevBuf mask;      // yb x xb round-edge factors of the cross-correlation
  DevBuf d_order, d_err, d_z0, d_maxerr, d_meas, d_bp;
  DevBuf d_applyjobs;  // FP32 operator mode: one ApplyJob per held-out tilt
  std::vector<size_t> bp_off;  // float offset of each tilt's geometry table in d_bp
  int ytiles = 0;
  cufftHandle rows_fwd_all = 0, rows_inv_all = 0, rows_fwd_one = 0, rows_inv_one = 0;
  cufftHandle cc_fwd = 0, cc_inv = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_kernels = 0;  // library kernels per replay
  double reproj_bytes = 0, reproj_fma = 0;  // per pass, over all held-out tilts
  std::vector<cudaEvent_t> events;  // 3 per held-out tilt when profiling
  bool use_graph = true;
  int method = 1;  // 1: banded operator with exact fallback; 0: exact gather only
  // FP16/BF16 modes: tensor-core apply of the operator to a 16-bit copy of the
  // corrected stack, exact FP32 fallback for row tiles the copy flags.
  int prec = MF_PREC_FP32;
  TcOpSet tcops;
  DevBuf corr16;    // nz x yb x xpitch 16-bit values
  DevBuf tflags;    // nz x ytiles
  DevBuf d_tcerr;   // pipeline error word of the tensor-core kernel
  TmaDesc imgmap;
  int tc_nb = 256, xpitch = 0;
  ~ProjAlignState();
};

struct TransformState {
  bool ready = false;
  int bin = 1, xb = 0, yb = 0;
  std::vector<float> pshx, pshy;
  DevBuf mask;  // yb x xb round-edge factors of the stretch correlations
};

}  // namespace mf

struct mf_series {
  mf_context* ctx = nullptr;
  int gpu = 0;
  int nx = 0, ny = 0, nz = 0;
  mf::DevBuf stack;  // pre-processed stack, nz x ny x nx
  mf::DevBuf stack_t;  // the same, column-major per tilt (nz x nx x ny)
  mf::DevBuf d_neg;    // nz ints: 1 when the pre-processed image holds a value below zero
  std::vector<float> file_angles;
  std::vector<float> angles;
  std::vector<float> sx, sy, rot;
  // FP16/BF16 modes: the shifts' FP64 accumulators (sx/sy hold their float values).
  // A float value the host changed replaces its accumulator at the next upload.
  std::vector<double> sx64, sy64;
  float angle_offset = 0.0f;
  mf::DevBuf d_sx, d_sy, d_rot, d_angles, d_sx64, d_sy64;
  mf_precision precision = MF_PREC_FP32;
  mf::TransformState tr;
  mf::ProjAlignState pa;
  bool shift64() const { return precision != MF_PREC_FP32; }
  double* dev_sx64() { return shift64() ? d_sx64.as<double>() : nullptr; }
  double* dev_sy64() { return shift64() ? d_sy64.as<double>() : nullptr; }
  int upload_params();
  // queues the shifts' copies to the host (and their accumulators in FP16/BF16
  // modes) without waiting
  int queue_download_shifts();
  int download_shifts();
};

namespace mf {
// Queued forms of the coarse stages (mf_series.cu): *_enqueue queues one series'
// work, its host results to the context's page-locked slot `slot`; *_finish reads
// them after the stream has been synchronised and updates the series.
struct TransformJob {
  std::vector<int> img_idx;  // tilt of each measured pair
  int np = 0;
  float2* h_sh = nullptr;    // page-locked: measured binned shift of each pair
};
struct AxisSearch {
  std::vector<float> cand;   // candidate axes
  AxisJob job;
};
constexpr int kOffsetCount = 31;  // tilt-angle offsets -15..15 degrees (FindOffset.cu:103-110)
struct OffsetJob {
  std::vector<int> first;    // first pair of each offset
  double* h_mom = nullptr;   // page-locked: 6 moments per (offset, pair)
};
int transform_enqueue(mf_series* s, int slot, TransformJob* job);
int transform_finish(mf_series* s, TransformJob* job, float* max_err);
int axis_enqueue(mf_series* s, float range, int num, int slot, AxisSearch* search);
int axis_finish(mf_series* s, AxisSearch* search, float* axis_out, float* scores_out);
int offset_enqueue(mf_series* s, int slot, OffsetJob* job);
int offset_finish(mf_series* s, OffsetJob* job, float* offset_out);
// Stage by stage over n series of one context, one wait per stage.
int transform_many(mf_series* const* ser, int n);
int tilt_axis_many(mf_series* const* ser, int n, float range, int num);
int coarse_align_many(mf_series* const* ser, int n, float pitch_angle, float offset);

int series_init(mf_series* s, mf_context* ctx, int nx, int ny, int nz, const float* file_angles);
int transform_doit(mf_series* s, float* max_err);
// scores_out (num floats, may be null): the score of every candidate
int tilt_axis(mf_series* s, float range, int num, float* axis_out, float* scores_out);
int find_offset(mf_series* s, float* offset_out);
int projalign_setup(mf_series* s, float zshift, int align_z, int nproj);
int projalign_doit(mf_series* s, float* max_err);
int coarse_align(mf_series* s, float pitch_angle, float offset);
int proj_align(mf_series* s, float zshift, int align_z, int nproj, int* passes);
int correct_stack_device(mf_series* s, int out_bin, float* d_out);
// groups (mf_batch.cu): series of one context and precision, of any shapes;
// align_z per series in the first form, shared in the second
int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift,
                 const int* align_z, int nproj, mf_group** out);
int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift, int align_z,
                 int nproj, mf_group** out);
int group_proj_align(mf_group* g, int* passes);
}  // namespace mf
