// Device-resident tilt series and the alignment stages that run on it.
#pragma once
#include <map>
#include <memory>

#include "mf_internal.hpp"

struct mf_context {
  mf::Context c;
  // scratch for the single-kernel entry points
  struct Scratch {
    mf::DevBuf a, b, c, d;
  } scratch;
  std::map<std::vector<long long>, cufftHandle> plans;
  ~mf_context();
  // Plan cache keyed by (kind, sizes, batch, layout); bound to the context stream.
  int plan(const std::vector<long long>& key, cufftHandle* out);
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
  DevBuf d_order, d_err, d_z0, d_maxerr, d_meas, d_rowflags, d_bp;
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
  float angle_offset = 0.0f;
  mf::DevBuf d_sx, d_sy, d_rot, d_angles;
  mf_precision precision = MF_PREC_FP32;
  mf::TransformState tr;
  mf::ProjAlignState pa;
  int upload_params();
  int download_shifts();
};

namespace mf {
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
// groups (mf_batch.cu): all series in `ctx`, same shape and precision
int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift, int align_z,
                 int nproj, mf_group** out);
int group_proj_align(mf_group* g, int* passes);
}  // namespace mf
