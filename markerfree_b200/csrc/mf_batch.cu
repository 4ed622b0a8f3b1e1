// Projection matching of many series in lockstep (a "group").
//
// Reference: Markerfree/src/method/ProjAlign.cpp:48-179 (Setup, DoIt, DoItBin) and
// Markerfree/src/main/Process.cpp:272-319 (mProjAlign, ProjAlignOnce), which align
// one series at a time.  Within a pass the held-out tilts of one series are
// sequential, so one series cannot fill a B200; series, however, are
// independent.  A group takes up to kMaxGroup series of one precision -- of any
// image size, tilt count and slab thickness -- and runs the k-th held-out tilt of
// every series together: each stage of the pass (correction, R-weight,
// re-projection, normalisation, filter, peak and parameter update,
// re-correction) is one launch over the whole group, every kernel reading its
// series' geometry and buffers from the series' GroupSeriesDev record.  cuFFT
// runs per series with the plan shapes of that series aligned alone.  A series
// with fewer tilts has no work in the last steps of a pass, and a per-series
// `active` flag lets each series leave ProjAlignOnce after its own number of
// passes.  Results per series are the same as when the series is aligned alone:
// the per-series arithmetic and its order are unchanged.
#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>

#include "mf_series.hpp"
#include "mf_xcorr.hpp"

using namespace mf;

namespace {

// Host-side state of one series of a group: its geometry, its work buffers of the
// pass and its cuFFT plans.
struct GroupMember {
  int nx = 0, ny = 0, nz = 0, n = 0, zt = 0;
  int bin = 1, xb = 0, yb = 0, pad = 0, cmp = 0, thick = 0, ytiles = 0, xpitch = 0;
  int out_x = 0, binx = 1, biny = 1;
  size_t bpix = 0, ppix = 0;
  DevBuf corr, scratch, reproj, cc, recorr, mpart, stats, ppart, corr16, tflags;
  const float* mask = nullptr;
  TmaDesc imgmap;
  std::vector<int> order;
  int op0 = 0;  // index of this series' first operator in the group's operator set
  cufftHandle rows_fwd_all = 0, rows_inv_all = 0;
  // the per-step transforms, one plan per side stream of the context
  static constexpr int kS = mf_context::kFftStreams;
  cufftHandle rows_fwd_one[kS] = {}, rows_inv_one[kS] = {}, cc_fwd[kS] = {}, cc_inv[kS] = {};
  // The parameters each tilt's corrected image was last made with (valid once a
  // pass has run), and this pass's start values of the shifts: a pass re-corrects
  // at its start only the tilts whose (shift, axis) changed since.
  bool corr_valid = false;
  std::vector<float> used_sx, used_sy, used_rot, start_sx, start_sy;
  int pre = 1;         // this pass's start: 0 nothing to redo, 1 every tilt, 2 one tilt
  int pre_tilt = -1;   // the tilt of pre == 2
};

}  // namespace

struct mf_group {
  mf_context* ctx = nullptr;
  std::vector<mf_series*> ser;
  int B = 0, prec = MF_PREC_FP32, nproj = 10;
  int nmax = 0;  // steps of a pass: the most held-out tilts of any series
  int nz_max = 0, xb_max = 0, yb_max = 0, pad_max = 0, cmp_max = 0, ytiles_max = 0;
  int ntiles_max = 0, rows_max = 0, tc_nb = 256;
  std::vector<std::unique_ptr<GroupMember>> m;
  // distinct re-projection operators (series with the same angles, size and slab
  // share theirs): per (series, step) entry op0 + k of the geometry list, its
  // operator's index; per operator, the bytes an apply reads and writes for the
  // images (per series) and reads of the operator itself (once per launch), MACs
  std::vector<int> opidx;
  std::vector<double> op_io, op_coef, op_mac;
  std::map<std::pair<int, int>, std::unique_ptr<DevBuf>> masks;  // per (xb, yb)
  std::vector<int> active;
  std::vector<float> z0;
  // device tables
  DevBuf d_ser, d_steps, d_active, d_bp, d_applyjobs, d_maxerr, d_z0, d_err, d_meas, d_tcerr;
  DevBuf d_full, d_pre;  // per series: re-correct every tilt at the pass start / the one tilt
  DevBuf d_order;
  ReprojOpSet ops;
  TcOpSet tcops;
  std::vector<TmaDesc> maps;               // per series
  std::vector<std::vector<TcJob>> tcjobs;  // per step: the series with a tilt at that step
  std::vector<cudaEvent_t> events;         // 3 per step when the context profiles
  ~mf_group() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
};

namespace mf {

// ProjAlign::Setsize (ProjAlign.cpp:48-125) and CorrTomoStack's sizes
// (CorrStack.cu:65-100) of one series.
static void member_geometry(GroupMember* M, const mf_series* s, int align_z) {
  M->nx = s->nx;
  M->ny = s->ny;
  M->nz = s->nz;
  M->n = s->nz - 1;
  const int bx = (int)((float)s->nx / 2048.0f + 0.5f), by = (int)((float)s->ny / 2048.0f + 0.5f);
  M->bin = std::max(1, std::max(bx, by));
  M->xb = s->nx / M->bin / 2 * 2;
  M->yb = s->ny / M->bin / 2 * 2;
  M->pad = (M->xb / 2 + 1) * 2;
  M->cmp = M->pad / 2;
  M->thick = align_z / M->bin / 2 * 2;
  const int pad_x = (s->nx / 2 + 1) * 2;
  M->out_x = (pad_x / 2 - 1) * 2;
  M->binx = M->out_x / M->xb;
  M->biny = s->ny / M->yb;
  M->bpix = (size_t)M->xb * M->yb;
  M->ppix = (size_t)M->pad * M->yb;
  M->ytiles = (M->yb + kApplyTileY - 1) / kApplyTileY;
  M->xpitch = (M->xb + 7) / 8 * 8;
}

static int group_setup(mf_group* g, float zshift, const int* align_z, int nproj) {
  StageTimer timer(&g->ctx->c, kStageSetup);
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B;
  if (nproj <= 0) return set_error(MF_ERR_ARG, "nproj must be > 0");
  g->nproj = nproj;
  g->m.clear();
  std::vector<ReprojGeom> geoms;
  std::vector<float> bp;
  std::vector<int> orders;
  std::vector<std::vector<GroupStepDev>> steps_b(B);
  for (int b = 0; b < B; ++b) {
    mf_series* s = g->ser[b];
    g->m.emplace_back(new GroupMember());
    GroupMember& M = *g->m.back();
    member_geometry(&M, s, align_z[b]);
    if (M.thick < 2)
      return set_error(MF_ERR_ARG, "series %d: slab thickness %d too small", b, M.thick);
    g->nz_max = std::max(g->nz_max, M.nz);
    g->nmax = std::max(g->nmax, M.n);
    g->xb_max = std::max(g->xb_max, M.xb);
    g->yb_max = std::max(g->yb_max, M.yb);
    g->pad_max = std::max(g->pad_max, M.pad);
    g->cmp_max = std::max(g->cmp_max, M.cmp);
    g->ytiles_max = std::max(g->ytiles_max, M.ytiles);
    g->ntiles_max = std::max(g->ntiles_max, (M.xb + kOpTileX - 1) / kOpTileX);
    g->rows_max = std::max(g->rows_max, M.nz * M.yb);
    // outward order and neighbour ranges (ProjAlign.cpp:151-176)
    const int nz = M.nz;
    M.zt = frame_idx_from_tilt(nz, s->angles.data(), 0.0f);
    std::vector<unsigned char> skip(nz, 1);
    skip[M.zt] = 0;
    std::vector<ReprojGeom> gb;
    for (int i = 1; i < nz; ++i) {
      for (int side = 0; side < 2; ++side) {
        int ip = side == 0 ? M.zt + i : M.zt - i;
        if (ip < 0 || ip >= nz) continue;
        int rg[2];
        find_proj_range(s->angles.data(), nz, skip.data(), ip, nproj, rg);
        if (rg[0] < 0 || rg[1] < 0)
          return set_error(MF_ERR_GEOMETRY,
                           "series %d: no already-aligned tilt within 20.5 degrees of tilt %d "
                           "(%.2f)",
                           b, ip, s->angles[ip]);
        ReprojGeom gm;
        reproj_geometry(s->angles.data(), ip, rg[0], rg[1], M.xb, M.yb, M.thick, &gm);
        gb.push_back(gm);
        skip[ip] = 0;
      }
    }
    if ((int)gb.size() != M.n)
      return set_error(MF_ERR_GEOMETRY, "series %d: %d held-out tilts instead of %d", b,
                       (int)gb.size(), M.n);
    MF_TRY(fill_bp_device(c, s->angles.data(), &gb, st));
    M.op0 = (int)geoms.size();
    for (const ReprojGeom& gm : gb) {
      GroupStepDev sd;
      sd.ip = gm.ip;
      sd.i0 = gm.i0;
      sd.nk = gm.nk;
      sd.ray_len = gm.ray_len;
      sd.thick = gm.thick;
      sd.bp_off = (int)bp.size();
      sd.fcos = gm.fcos;
      sd.fsin = gm.fsin;
      bp.insert(bp.end(), gm.bp.begin(), gm.bp.end());
      steps_b[b].push_back(sd);
      M.order.push_back(gm.ip);
      geoms.push_back(gm);
    }
  }
  const int nmax = g->nmax;
  // steps table [k][b]; a series without a tilt at step k gets ip = -1
  std::vector<GroupStepDev> steps((size_t)nmax * B);
  for (int k = 0; k < nmax; ++k)
    for (int b = 0; b < B; ++b) {
      GroupStepDev sd{};
      sd.ip = -1;
      if (k < (int)steps_b[b].size()) sd = steps_b[b][k];
      steps[(size_t)k * B + b] = sd;
    }
  // per-series buffers
  for (int b = 0; b < B; ++b) {
    GroupMember& M = *g->m[b];
    MF_TRY(M.corr.alloc(sizeof(float) * M.bpix * M.nz));
    MF_TRY(M.scratch.alloc(sizeof(float) * M.ppix * M.nz));
    MF_TRY(M.reproj.alloc(sizeof(float) * M.bpix));
    MF_TRY(M.cc.alloc(sizeof(float) * M.ppix * 2));
    MF_TRY(M.recorr.alloc(sizeof(float) * M.ppix));
    MF_TRY(M.mpart.alloc(sizeof(double2) * moment_parts(M.yb) * 2));
    MF_TRY(M.stats.alloc(sizeof(float2) * 2));
    MF_TRY(M.ppart.alloc(sizeof(float2) * kPeakParts));
    auto key = std::make_pair(M.xb, M.yb);
    auto it = g->masks.find(key);
    if (it == g->masks.end()) {
      std::unique_ptr<DevBuf> mk(new DevBuf());
      MF_TRY(mk->alloc(sizeof(float) * M.bpix));
      MF_TRY(make_round_mask(c, M.xb, M.yb, (float)((M.pad / 2 - 1) * 2) * 0.5f,
                             (float)M.yb * 0.5f, (float)M.pad, (float)M.yb, 4.0f,
                             mk->as<float>(), st));
      it = g->masks.emplace(key, std::move(mk)).first;
    }
    M.mask = it->second->as<float>();
    if (g->prec != MF_PREC_FP32) MF_TRY(M.corr16.alloc((size_t)2 * M.xpitch * M.yb * M.nz));
    MF_TRY(M.tflags.alloc(sizeof(int) * (size_t)M.nz * M.ytiles * kFlagParts));
    for (int z : M.order) orders.push_back(z);
  }
  MF_TRY(g->d_steps.alloc(sizeof(GroupStepDev) * steps.size()));
  MF_TRY(g->d_order.alloc(sizeof(int) * std::max<size_t>(orders.size(), 1)));
  MF_TRY(g->d_bp.alloc(sizeof(float) * std::max<size_t>(bp.size(), 1)));
  MF_TRY(g->d_active.alloc(sizeof(int) * B));
  MF_TRY(g->d_full.alloc(sizeof(int) * B));
  MF_TRY(g->d_pre.alloc(sizeof(GroupStepDev) * B));
  MF_TRY(g->d_maxerr.alloc(sizeof(float) * B));
  MF_TRY(g->d_z0.alloc(sizeof(float) * B));
  MF_TRY(g->d_err.alloc(sizeof(float) * g->nz_max * B));
  MF_TRY(g->d_meas.alloc(sizeof(float) * 2 * g->nz_max * B));
  MF_TRY(g->d_tcerr.alloc(sizeof(int)));
  MF_TRY(g->d_ser.alloc(sizeof(GroupSeriesDev) * B));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_steps.p, steps.data(), sizeof(GroupStepDev) * steps.size(),
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_order.p, orders.data(), sizeof(int) * orders.size(),
                                cudaMemcpyHostToDevice, st));
  if (!bp.empty())
    MF_CHECK_CUDA(cudaMemcpyAsync(g->d_bp.p, bp.data(), sizeof(float) * bp.size(),
                                  cudaMemcpyHostToDevice, st));
  g->z0.assign(B, zshift);
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_z0.p, g->z0.data(), sizeof(float) * B, cudaMemcpyHostToDevice,
                                st));
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_err.p, 0, sizeof(float) * g->nz_max * B, st));
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_meas.p, 0, sizeof(float) * 2 * g->nz_max * B, st));
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_tcerr.p, 0, sizeof(int), st));
  std::vector<GroupSeriesDev> sd(B);
  size_t order_off = 0;
  for (int b = 0; b < B; ++b) {
    mf_series* s = g->ser[b];
    GroupMember& M = *g->m[b];
    GroupSeriesDev& d = sd[b];
    memset(&d, 0, sizeof(d));
    d.stack = s->stack.as<float>();
    d.stack_t = s->stack_t.as<float>();
    d.sx = s->d_sx.as<float>();
    d.sy = s->d_sy.as<float>();
    d.sx64 = s->dev_sx64();
    d.sy64 = s->dev_sy64();
    d.rot = s->d_rot.as<float>();
    d.angles = s->d_angles.as<float>();
    d.z0 = g->d_z0.as<float>() + b;
    d.err = g->d_err.as<float>() + (size_t)b * g->nz_max;
    d.meas = g->d_meas.as<float>() + (size_t)b * 2 * g->nz_max;
    d.corr = M.corr.as<float>();
    d.order = g->d_order.as<int>() + order_off;
    order_off += M.order.size();
    d.zt = M.zt;
    d.n = M.n;
    d.nx = M.nx;
    d.ny = M.ny;
    d.nz = M.nz;
    d.bin = M.bin;
    d.out_x = M.out_x;
    d.binx = M.binx;
    d.biny = M.biny;
    d.xb = M.xb;
    d.yb = M.yb;
    d.pad = M.pad;
    d.cmp = M.cmp;
    d.ytiles = M.ytiles;
    d.xpitch = M.xpitch;
    d.bpix = M.bpix;
    d.ppix = M.ppix;
    d.scratch = M.scratch.as<float>();
    d.reproj = M.reproj.as<float>();
    d.cc = M.cc.as<float>();
    d.recorr = M.recorr.as<float>();
    d.mask = M.mask;
    d.mpart = M.mpart.as<double2>();
    d.stats = M.stats.as<float2>();
    d.ppart = M.ppart.as<float2>();
    d.corr16 = M.corr16.p;
    d.tflags = M.tflags.as<int>();
  }
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_ser.p, sd.data(), sizeof(GroupSeriesDev) * B,
                                cudaMemcpyHostToDevice, st));
  // re-projection operators of every (series, step): geometry index op0 + k.
  // Series of one acquisition scheme have identical geometries (same angles, size,
  // slab): each distinct one is built once and shared.
  std::vector<ReprojGeom> uniq;
  g->opidx.assign(geoms.size(), 0);
  {
    auto bits = [](float v) {
      uint32_t u;
      memcpy(&u, &v, 4);
      return u;
    };
    std::map<std::vector<uint32_t>, int> seen;
    for (size_t i = 0; i < geoms.size(); ++i) {
      const ReprojGeom& gm = geoms[i];
      std::vector<uint32_t> key = {(uint32_t)gm.xb,  (uint32_t)gm.yb, (uint32_t)gm.thick,
                                   (uint32_t)gm.ip,  (uint32_t)gm.i0, (uint32_t)gm.i1,
                                   (uint32_t)gm.nk,  (uint32_t)gm.ray_len, bits(gm.fcos),
                                   bits(gm.fsin)};
      for (float v : gm.bp) key.push_back(bits(v));
      auto it = seen.find(key);
      if (it == seen.end()) {
        it = seen.emplace(std::move(key), (int)uniq.size()).first;
        uniq.push_back(gm);
      }
      g->opidx[i] = it->second;
    }
  }
  g->tcjobs.assign(nmax, {});
  if (g->prec != MF_PREC_FP32) {
    MF_TRY(build_reproj_tc_ops_any(c, uniq, g->prec, &g->tcops, st));
    for (const TcOpView& v : g->tcops.ops) {
      g->op_io.push_back(2.0 * v.xb * v.yb * v.nk + 4.0 * v.xb * v.yb);
      g->op_coef.push_back((double)v.nchunks * kTcM * kTcK * 2);
      g->op_mac.push_back((double)v.nchunks * kTcM * kTcK * v.yb);
    }
    g->maps.assign(B, TmaDesc());
    for (int b = 0; b < B; ++b) {
      const GroupMember& M = *g->m[b];
      for (int k = 0; k < M.n; ++k) {
        const TcOpView& v = g->tcops.ops[g->opidx[M.op0 + k]];
        g->tcjobs[k].push_back(TcJob{v.xt, v.colvalid, M.reproj.as<float>(), b, b, M.xb, M.yb,
                                     0, 0});
      }
    }
    // tile rows: timed on the first step, on zeroed 16-bit stacks (the launches
    // only write the re-projection buffers, which every pass overwrites)
    for (int b = 0; b < B; ++b) {
      GroupMember& M = *g->m[b];
      MF_CHECK_CUDA(cudaMemsetAsync(M.corr16.p, 0, M.corr16.bytes, st));
    }
    MF_TRY(tc_autotune_rows(
        c, g->xb_max, g->yb_max, B, g->prec,
        [&](int nb) -> int {
          for (int b = 0; b < B; ++b) {
            GroupMember& M = *g->m[b];
            MF_TRY(tc_image_map(M.corr16.p, g->prec, M.xb, M.xpitch, M.yb, M.nz, nb, &g->maps[b]));
          }
          return launch_reproject_tc_group(c, g->tcops, g->tcjobs[0].data(),
                                           (int)g->tcjobs[0].size(), nullptr, g->maps.data(), B,
                                           nb, g->d_tcerr.as<int>(), st);
        },
        g->d_tcerr.as<int>(), &g->tc_nb, st));
    MF_TRY(tc_prepare(c, g->tc_nb));
    for (int b = 0; b < B; ++b) {
      GroupMember& M = *g->m[b];
      MF_TRY(tc_image_map(M.corr16.p, g->prec, M.xb, M.xpitch, M.yb, M.nz, g->tc_nb, &g->maps[b]));
    }
    MF_CHECK_CUDA(cudaMemsetAsync(g->d_tcerr.p, 0, sizeof(int), st));
  } else {
    MF_TRY(build_reproj_ops_any(c, uniq, &g->ops, st));
    MF_TRY(prepare_apply_group(c));  // before any capture of a pass
    for (const ReprojOpView& v : g->ops.ops) {
      g->op_io.push_back(4.0 * v.xb * v.yb * (v.nk + 1));
      g->op_coef.push_back((double)v.total_rows * (kOpTileX * 4 + 8));
      g->op_mac.push_back((double)v.yb * v.total_rows * kOpTileX);
    }
    std::vector<ApplyJob> jobs((size_t)nmax * B);
    for (int k = 0; k < nmax; ++k)
      for (int b = 0; b < B; ++b) {
        const GroupMember& M = *g->m[b];
        ApplyJob J{};
        if (k < M.n) {
          const ReprojOpView& v = g->ops.ops[g->opidx[M.op0 + k]];
          J.tiles = v.tiles;
          J.colvalid = v.colvalid;
          J.corr = M.corr.as<float>();
          J.out = M.reproj.as<float>();
          J.xb = M.xb;
          J.yb = M.yb;
          J.ntiles = v.ntiles;
        }
        jobs[(size_t)k * B + b] = J;
      }
    MF_TRY(g->d_applyjobs.alloc(sizeof(ApplyJob) * jobs.size()));
    MF_CHECK_CUDA(cudaMemcpyAsync(g->d_applyjobs.p, jobs.data(), sizeof(ApplyJob) * jobs.size(),
                                  cudaMemcpyHostToDevice, st));
  }
  // FFT plans (cached per context).  The same plan shapes as the series' own pass,
  // executed once per series: a plan batched over the group may round
  // differently, and a different rounding can flip a near-tied decision later
  // (tilt-axis candidates, nearest-neighbour re-correction), so per-series
  // execution keeps each result identical to the series aligned alone.
  mf_context* ctx = g->ctx;
  for (int b = 0; b < B; ++b) {
    GroupMember& M = *g->m[b];
    MF_TRY(ctx->plan({0, M.xb, M.yb, (long long)M.nz * M.yb}, &M.rows_fwd_all));
    MF_TRY(ctx->plan({1, M.xb, M.yb, (long long)M.nz * M.yb}, &M.rows_inv_all));
    for (int i = 0; i < mf_context::kFftStreams; ++i) {
      MF_TRY(ctx->plan({0, M.xb, M.yb, (long long)M.yb, i}, &M.rows_fwd_one[i]));
      MF_TRY(ctx->plan({1, M.xb, M.yb, (long long)M.yb, i}, &M.rows_inv_one[i]));
      MF_TRY(ctx->plan({2, M.xb, M.yb, 2, i}, &M.cc_fwd[i]));
      MF_TRY(ctx->plan({3, M.xb, M.yb, 1, i}, &M.cc_inv[i]));
    }
  }
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// One projection-matching pass over the active series (the group form of
// pa_enqueue in mf_series.cu).  cuFFT runs only for the series that take part in
// a stage (active, and with a held-out tilt at the step).
static int group_enqueue(mf_group* g) {
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B, nmax = g->nmax;
  const bool tc = g->prec != MF_PREC_FP32;
  const GroupSeriesDev* ser = g->d_ser.as<GroupSeriesDev>();
  const GroupStepDev* steps = g->d_steps.as<GroupStepDev>();
  const int* active = g->d_active.as<int>();
  std::vector<TcJob> jobs;
  // A per-step FFT stage: the transforms of the series that take part run on the
  // context's side streams, forked from the stream after the work queued so far
  // and joined back before the next kernel; each series' own plans, so the
  // results are those of the transforms run one after another.
  mf_context* ctx = g->ctx;
  const int nfs = mf_context::kFftStreams;
  // (k < 0: the series whose pass start re-corrects one tilt take part)
  auto fft_stage = [&](int k, const std::function<int(GroupMember&, int)>& exec) -> int {
    MF_CHECK_CUDA(cudaEventRecord(ctx->fork_ev, st));
    int used = 0;
    for (int b = 0; b < B; ++b) {
      if (!g->active[b]) continue;
      if (k < 0 ? g->m[b]->pre != 2 : k >= g->m[b]->n) continue;
      const int slot = used % nfs;
      if (used < nfs) MF_CHECK_CUDA(cudaStreamWaitEvent(ctx->aux[slot], ctx->fork_ev, 0));
      MF_TRY(exec(*g->m[b], slot));
      ++used;
    }
    for (int i = 0; i < std::min(used, nfs); ++i) {
      MF_CHECK_CUDA(cudaEventRecord(ctx->join_ev[i], ctx->aux[i]));
      MF_CHECK_CUDA(cudaStreamWaitEvent(st, ctx->join_ev[i], 0));
    }
    return MF_OK;
  };
  // CorrTomoStack::DoIt at the pass start: every tilt of the series whose
  // parameters changed beyond one tilt (d_full), the one changed tilt of the
  // others (d_pre; the same kernels and plans as a step's re-correction), nothing
  // for a series whose corrected stack is current
  const int* full = g->d_full.as<int>();
  GroupCorrArgs ca{ser, nullptr, full, g->nz_max, 1};
  MF_TRY(launch_correct_group(c, ca, B, g->xb_max, g->yb_max, st));
  for (int b = 0; b < B; ++b)
    if (g->active[b] && g->m[b]->pre == 1) {
      float* sb = g->m[b]->scratch.as<float>();
      MF_CHECK_CUFFT(cufftExecR2C(g->m[b]->rows_fwd_all, sb, (cufftComplex*)sb));
    }
  MF_TRY(launch_rweight_group(c, ser, nullptr, full, B, g->cmp_max, g->rows_max, st));
  for (int b = 0; b < B; ++b)
    if (g->active[b] && g->m[b]->pre == 1)
      MF_CHECK_CUFFT(cufftExecC2R(g->m[b]->rows_inv_all,
                                  (cufftComplex*)g->m[b]->scratch.as<float>(),
                                  g->m[b]->corr.as<float>()));
  if (tc)
    MF_TRY(launch_to_half_group(c, ser, nullptr, full, B, g->nz_max, g->ytiles_max, g->prec,
                                st));
  else
    MF_TRY(launch_flag_tiles_group(c, ser, nullptr, full, B, g->nz_max, g->ytiles_max, st));
  bool any_one = false;
  for (int b = 0; b < B; ++b) any_one |= g->active[b] && g->m[b]->pre == 2;
  if (any_one) {
    const GroupStepDev* pre = g->d_pre.as<GroupStepDev>();
    GroupCorrArgs rc{ser, pre, active, g->nz_max, 1};
    MF_TRY(launch_correct_group(c, rc, B, g->xb_max, g->yb_max, st));
    MF_TRY(fft_stage(-1, [&](GroupMember& M, int i) -> int {
      float* rb = M.recorr.as<float>();
      MF_CHECK_CUFFT(cufftExecR2C(M.rows_fwd_one[i], rb, (cufftComplex*)rb));
      return MF_OK;
    }));
    MF_TRY(launch_rweight_group(c, ser, pre, active, B, g->cmp_max, g->yb_max, st));
    MF_TRY(fft_stage(-1, [&](GroupMember& M, int i) -> int {
      MF_CHECK_CUFFT(cufftExecC2R(M.rows_inv_one[i], (cufftComplex*)M.recorr.as<float>(),
                                  M.corr.as<float>() + (size_t)M.pre_tilt * M.bpix));
      return MF_OK;
    }));
    if (tc)
      MF_TRY(launch_to_half_group(c, ser, pre, active, B, g->nz_max, g->ytiles_max, g->prec,
                                  st));
    else
      MF_TRY(launch_flag_tiles_group(c, ser, pre, active, B, g->nz_max, g->ytiles_max, st));
  }
  MF_TRY(fit_z0_group(c, ser, active, B, st));
  const bool prof = c->profiling && (int)g->events.size() >= 3 * nmax;
  for (int k = 0; k < nmax; ++k) {
    const GroupStepDev* sk = steps + (size_t)k * B;
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k], st));
    if (tc) {
      jobs.clear();
      for (const TcJob& J : g->tcjobs[k])
        if (g->active[J.series]) jobs.push_back(J);
      MF_TRY(launch_reproject_tc_group(c, g->tcops, jobs.data(), (int)jobs.size(), active,
                                       g->maps.data(), B, g->tc_nb, g->d_tcerr.as<int>(), st));
      MF_TRY(launch_reproject_exact_group(c, ser, sk, active, B, g->xb_max, g->ytiles_max,
                                          g->d_bp.as<float>(), true, nullptr, st));
    } else {
      MF_TRY(launch_reproject_apply_group(c, g->ops, g->d_applyjobs.as<ApplyJob>() + (size_t)k * B,
                                          active, B, g->ntiles_max, g->yb_max, st));
      MF_TRY(launch_reproject_exact_group(c, ser, sk, active, B, g->xb_max, g->ytiles_max,
                                          g->d_bp.as<float>(), true, nullptr, st));
    }
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k + 1], st));
    // MeaAlignProj for every series: PANorm both images, FFT, filter, inverse, peak
    MF_TRY(norm_mask_pad_group(c, ser, sk, active, B, g->xb_max, g->yb_max, g->pad_max, st));
    MF_TRY(fft_stage(k, [&](GroupMember& M, int i) -> int {
      float* cb = M.cc.as<float>();
      MF_CHECK_CUFFT(cufftExecR2C(M.cc_fwd[i], cb, (cufftComplex*)cb));
      return MF_OK;
    }));
    MF_TRY(xcorr_filter_group(c, ser, sk, active, B, g->cmp_max, g->yb_max, 500.0f, st));
    MF_TRY(fft_stage(k, [&](GroupMember& M, int i) -> int {
      float* mb = M.cc.as<float>() + M.ppix;
      MF_CHECK_CUFFT(cufftExecC2R(M.cc_inv[i], (cufftComplex*)mb, mb));
      return MF_OK;
    }));
    MF_TRY(pa_peak_update_group(c, ser, sk, active, B, st));
    // re-correct the aligned tilt of every series (mCorrectProj)
    GroupCorrArgs rc{ser, sk, active, g->nz_max, 1};
    MF_TRY(launch_correct_group(c, rc, B, g->xb_max, g->yb_max, st));
    MF_TRY(fft_stage(k, [&](GroupMember& M, int i) -> int {
      float* rb = M.recorr.as<float>();
      MF_CHECK_CUFFT(cufftExecR2C(M.rows_fwd_one[i], rb, (cufftComplex*)rb));
      return MF_OK;
    }));
    MF_TRY(launch_rweight_group(c, ser, sk, active, B, g->cmp_max, g->yb_max, st));
    // the inverse row transforms write the re-corrected tilt into its place in
    // the corrected stack (nothing reads the old one after the measurement)
    MF_TRY(fft_stage(k, [&](GroupMember& M, int i) -> int {
      MF_CHECK_CUFFT(cufftExecC2R(M.rows_inv_one[i], (cufftComplex*)M.recorr.as<float>(),
                                  M.corr.as<float>() + (size_t)M.order[k] * M.bpix));
      return MF_OK;
    }));
    if (tc)
      MF_TRY(launch_to_half_group(c, ser, sk, active, B, g->nz_max, g->ytiles_max, g->prec, st));
    else
      MF_TRY(launch_flag_tiles_group(c, ser, sk, active, B, g->nz_max, g->ytiles_max, st));
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k + 2], st));
  }
  MF_TRY(max_err_group(c, ser, active, B, g->d_maxerr.as<float>(), st));
  return MF_OK;
}

// One pass over the series with active[b] != 0; max_err[b] receives each active
// series' largest measured shift (inactive entries are left as they are).  The
// pass is launched eagerly: its cuFFT calls depend on which series take part.
static int group_doit(mf_group* g, const int* active, float* max_err) {
  StageTimer timer(&g->ctx->c, kStagePass);
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B;
  g->active.assign(active, active + B);
  for (int b = 0; b < B; ++b) MF_TRY(g->ser[b]->upload_params());
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_active.p, g->active.data(), sizeof(int) * B,
                                cudaMemcpyHostToDevice, st));
  // what the pass start has to re-correct, per active series: the tilts whose
  // (shift, axis) differ from those their corrected image was made with
  std::vector<int> full(B, 0);
  std::vector<GroupStepDev> pre(B);
  for (int b = 0; b < B; ++b) {
    GroupMember& M = *g->m[b];
    const mf_series* s = g->ser[b];
    memset(&pre[b], 0, sizeof(GroupStepDev));
    pre[b].ip = -1;
    if (!active[b]) continue;
    M.pre = 1;
    if (M.corr_valid) {
      int changed = 0, last = -1;
      for (int i = 0; i < M.nz; ++i)
        if (s->sx[i] != M.used_sx[i] || s->sy[i] != M.used_sy[i] || s->rot[i] != M.used_rot[i]) {
          ++changed;
          last = i;
        }
      M.pre = changed == 0 ? 0 : changed == 1 ? 2 : 1;
      M.pre_tilt = last;
    }
    full[b] = M.pre == 1;
    if (M.pre == 2) pre[b].ip = M.pre_tilt;
    M.start_sx = s->sx;
    M.start_sy = s->sy;
  }
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_full.p, full.data(), sizeof(int) * B, cudaMemcpyHostToDevice,
                                st));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_pre.p, pre.data(), sizeof(GroupStepDev) * B,
                                cudaMemcpyHostToDevice, st));
  while (c->profiling && (int)g->events.size() < 3 * g->nmax) {
    cudaEvent_t e;
    MF_CHECK_CUDA(cudaEventCreate(&e));
    g->events.push_back(e);
  }
  MF_TRY(group_enqueue(g));
  std::vector<float> me(B);
  int tcerr = 0;
  MF_CHECK_CUDA(cudaMemcpyAsync(me.data(), g->d_maxerr.p, sizeof(float) * B,
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->z0.data(), g->d_z0.p, sizeof(float) * B,
                                cudaMemcpyDeviceToHost, st));
  if (g->prec != MF_PREC_FP32)
    MF_CHECK_CUDA(cudaMemcpyAsync(&tcerr, g->d_tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  for (int b = 0; b < B; ++b) MF_TRY(g->ser[b]->queue_download_shifts());
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  if (tcerr != 0)
    return set_error(MF_ERR_CUDA, "tensor-core re-projection pipeline stalled (code %d)", tcerr);
  for (int b = 0; b < B; ++b)
    if (active[b]) {
      max_err[b] = me[b];
      g->ser[b]->pa.z0 = g->z0[b];
      // every held-out tilt was re-corrected at its step with its final shift; the
      // zero tilt keeps the image made at the pass start, with the start shift
      GroupMember& M = *g->m[b];
      const mf_series* s = g->ser[b];
      M.used_sx = s->sx;
      M.used_sy = s->sy;
      M.used_rot = s->rot;
      M.used_sx[M.zt] = M.start_sx[M.zt];
      M.used_sy[M.zt] = M.start_sy[M.zt];
      M.corr_valid = true;
    }
  // compulsory bytes and MACs of this pass's re-projection launches: per step, the
  // images and output of every series taking part, each distinct operator once
  double pass_bytes = 0, pass_mac = 0;
  std::vector<int> used;
  for (int k = 0; k < g->nmax; ++k) {
    used.clear();
    for (int b = 0; b < B; ++b) {
      if (!active[b] || k >= g->m[b]->n) continue;
      const int o = g->opidx[g->m[b]->op0 + k];
      pass_bytes += g->op_io[o];
      pass_mac += g->op_mac[o];
      if (std::find(used.begin(), used.end(), o) == used.end()) {
        used.push_back(o);
        pass_bytes += g->op_coef[o];
      }
    }
  }
  if (c->profiling && (int)g->events.size() >= 3 * g->nmax) {
    // stage times of this pass: [0] re-projection launches (one per step for the
    // whole group), [2] the rest of each step; bytes and MACs of the active series
    for (int k = 0; k < g->nmax; ++k) {
      float a = 0.0f, b2 = 0.0f;
      MF_CHECK_CUDA(cudaEventElapsedTime(&a, g->events[3 * k], g->events[3 * k + 1]));
      MF_CHECK_CUDA(cudaEventElapsedTime(&b2, g->events[3 * k + 1], g->events[3 * k + 2]));
      c->stage[0] += a;
      c->stage[2] += b2;
    }
    c->stage[1] += g->nmax;
    c->stage[3] += 1;
    c->stage[4] += pass_bytes;
    c->stage[5] += pass_mac;
  }
  return MF_OK;
}

// Process::mProjAlign + ProjAlignOnce (Process.cpp:272-319) for every series of
// the group.  Each series follows its own break rule; a pass runs the series that
// are still inside the current ProjAlignOnce loop.
int group_proj_align(mf_group* g, int* passes) {
  const int B = g->B;
  std::vector<int> np(B, 0);
  // ResetShift (Process.cpp:321-327); the axis found by the coarse stage is kept
  for (int b = 0; b < B; ++b) {
    std::fill(g->ser[b]->sx.begin(), g->ser[b]->sx.end(), 0.0f);
    std::fill(g->ser[b]->sy.begin(), g->ser[b]->sy.end(), 0.0f);
  }
  auto once = [&]() -> int {
    std::vector<int> it(B, 0), act(B, 1);
    std::vector<float> last(B, 0.0f), e(B, 0.0f);
    while (true) {
      int any = 0;
      for (int b = 0; b < B; ++b) any |= act[b];
      if (!any) break;
      MF_TRY(group_doit(g, act.data(), e.data()));
      for (int b = 0; b < B; ++b) {
        if (!act[b]) continue;
        np[b]++;
        if (it[b] == 0) {
          last[b] = e[b];
        } else if (e[b] <= last[b]) {
          if (e[b] < 2.0f) act[b] = 0;
          last[b] = e[b];
        }
        if (++it[b] >= 10) act[b] = 0;
      }
    }
    return MF_OK;
  };
  MF_TRY(once());
  for (int i = 1; i <= 4; ++i) {
    MF_TRY(tilt_axis_many(g->ser.data(), B, 20.0f / i, 100));
    if (i == 1) MF_TRY(once());
  }
  MF_TRY(once());
  if (passes)
    for (int b = 0; b < B; ++b) passes[b] = np[b];
  return MF_OK;
}

int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift,
                 const int* align_z, int nproj, mf_group** out) {
  if (!out) return set_error(MF_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (!ctx || !series || !align_z || nser < 1 || nser > kMaxGroup)
    return set_error(MF_ERR_ARG, "a group holds 1..%d series (got %d)", kMaxGroup, nser);
  for (int b = 0; b < nser; ++b) {
    const mf_series* s = series[b];
    if (!s) return set_error(MF_ERR_ARG, "null series %d", b);
    if (s->ctx != ctx) return set_error(MF_ERR_ARG, "series %d belongs to another context", b);
    if (s->gpu != ctx->c.gpu) return set_error(MF_ERR_ARG, "series %d is on another GPU", b);
    if (s->precision != series[0]->precision)
      return set_error(MF_ERR_ARG, "series %d differs in precision from series 0", b);
  }
  mf_group* g = new mf_group();
  g->ctx = ctx;
  g->ser.assign(series, series + nser);
  g->B = nser;
  g->prec = series[0]->precision;
  int rc = group_setup(g, zshift, align_z, nproj);
  if (rc != MF_OK) {
    delete g;
    return rc;
  }
  *out = g;
  return MF_OK;
}

int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift, int align_z,
                 int nproj, mf_group** out) {
  std::vector<int> az(std::max(nser, 0), align_z);
  return group_create(ctx, series, nser, zshift, az.data(), nproj, out);
}

}  // namespace mf

// ---------------------------------------------------------------------------
#define MF_GUARD_BEGIN try {
#define MF_GUARD_END                                                      \
  }                                                                       \
  catch (const std::bad_alloc&) {                                         \
    return set_error(MF_ERR_NOMEM, "host allocation failed");             \
  }                                                                       \
  catch (...) {                                                           \
    return set_error(MF_ERR_STATE, "unexpected exception in the library"); \
  }

// Process::DoIt minus file I/O (Process.cpp:34-92) for n series given by their
// device buffers, sizes and slab thicknesses: every series is uploaded and
// pre-processed, coarse-aligned stage by stage with the others of its group of
// up to kMaxGroup, projection-matched with them in lockstep, then corrected into
// its output buffer.
static int align_batch(mf_context* ctx, int n, const float* const* d_raw, const int* nx,
                       const int* ny, const int* nz, const float* const* file_angles,
                       const int* align_z, const mf_options* opt, mf_align_param* params,
                       float* const* d_out, int* passes) {
  if (!ctx || n < 1 || !d_raw || !file_angles || !opt || !params)
    return set_error(MF_ERR_ARG, "null argument");
  if (opt->nproj <= 0) return set_error(MF_ERR_ARG, "nProj must be > 0.");
  if (opt->out_bin < 1) return set_error(MF_ERR_ARG, "output binning must be >= 1");
  if (opt->precision != MF_PREC_FP32 && opt->precision != MF_PREC_BF16 &&
      opt->precision != MF_PREC_FP16)
    return set_error(MF_ERR_ARG, "unknown precision %d", opt->precision);
  std::vector<mf_series*> ser(n, nullptr);
  auto cleanup = [&]() {
    for (mf_series* s : ser) mf_series_destroy(s);
  };
  int rc = MF_OK;
  for (int i = 0; i < n && rc == MF_OK; ++i) {
    rc = mf_series_create_device(ctx, d_raw[i], nx[i], ny[i], nz[i], file_angles[i], &ser[i]);
    if (rc == MF_OK) ser[i]->precision = (mf_precision)opt->precision;
  }
  const bool align = opt->align_z != 0;
  for (int g0 = 0; g0 < n && rc == MF_OK && align; g0 += kMaxGroup)
    rc = coarse_align_many(ser.data() + g0, std::min(kMaxGroup, n - g0), opt->pitch_angle,
                           opt->offset);
  for (int g0 = 0; g0 < n && rc == MF_OK && align; g0 += kMaxGroup) {
    const int m = std::min(kMaxGroup, n - g0);
    mf_group* g = nullptr;
    rc = group_create(ctx, ser.data() + g0, m, opt->zshift, align_z + g0, opt->nproj, &g);
    if (rc == MF_OK) rc = group_proj_align(g, passes ? passes + g0 : nullptr);
    delete g;
  }
  if (!align && passes)
    for (int i = 0; i < n; ++i) passes[i] = 0;
  for (int i = 0; i < n && rc == MF_OK; ++i) {
    if (d_out && d_out[i]) rc = correct_stack_device(ser[i], opt->out_bin, d_out[i]);
    if (rc == MF_OK) rc = mf_series_get_param(ser[i], &params[i]);
  }
  if (rc == MF_OK && cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
    rc = set_error(MF_ERR_CUDA, "stream synchronize failed");
  cleanup();
  return rc;
}

extern "C" {

MF_API int mf_group_create(mf_series* const* series, int n, float zshift, int align_z, int nproj,
                           mf_group** out) {
  MF_GUARD_BEGIN
  if (!series || n < 1 || !series[0]) return set_error(MF_ERR_ARG, "no series");
  mf_context* ctx = series[0]->ctx;
  MF_CHECK_CUDA(cudaSetDevice(ctx->c.gpu));
  set_alloc_stream(ctx->c.stream);
  return group_create(ctx, series, n, zshift, align_z, nproj, out);
  MF_GUARD_END
}

MF_API void mf_group_destroy(mf_group* g) {
  if (!g) return;
  cudaSetDevice(g->ctx->c.gpu);
  delete g;
}

MF_API int mf_group_doit(mf_group* g, const int* active, float* max_err) {
  MF_GUARD_BEGIN
  if (!g || !active || !max_err) return set_error(MF_ERR_ARG, "null argument");
  MF_CHECK_CUDA(cudaSetDevice(g->ctx->c.gpu));
  set_alloc_stream(g->ctx->c.stream);
  return group_doit(g, active, max_err);
  MF_GUARD_END
}

MF_API int mf_group_proj_align(mf_group* g, int* passes) {
  MF_GUARD_BEGIN
  if (!g) return set_error(MF_ERR_ARG, "null group");
  MF_CHECK_CUDA(cudaSetDevice(g->ctx->c.gpu));
  set_alloc_stream(g->ctx->c.stream);
  return group_proj_align(g, passes);
  MF_GUARD_END
}

MF_API int mf_align_many_device(mf_context* ctx, int n, const float* const* d_raw, int nx, int ny,
                                int nz, const float* const* file_angles, const mf_options* opt,
                                mf_align_param* params, float* const* d_out, int* passes) {
  MF_GUARD_BEGIN
  if (!ctx || n < 1 || !opt) return set_error(MF_ERR_ARG, "null argument");
  std::vector<int> vx(n, nx), vy(n, ny), vz(n, nz), az(n, opt->align_z);
  return align_batch(ctx, n, d_raw, vx.data(), vy.data(), vz.data(), file_angles, az.data(), opt,
                     params, d_out, passes);
  MF_GUARD_END
}

MF_API int mf_align_batch_device(mf_context* ctx, int n, const mf_series_desc* series,
                                 const mf_options* opt, mf_align_param* params, int* passes) {
  MF_GUARD_BEGIN
  if (!ctx || n < 1 || !series || !opt) return set_error(MF_ERR_ARG, "null argument");
  std::vector<const float*> raw(n), ang(n);
  std::vector<float*> out(n);
  std::vector<int> vx(n), vy(n), vz(n), az(n);
  for (int i = 0; i < n; ++i) {
    raw[i] = series[i].d_raw;
    ang[i] = series[i].file_angles;
    out[i] = series[i].d_out;
    vx[i] = series[i].nx;
    vy[i] = series[i].ny;
    vz[i] = series[i].nz;
    az[i] = series[i].align_z != 0 ? series[i].align_z : opt->align_z;
  }
  return align_batch(ctx, n, raw.data(), vx.data(), vy.data(), vz.data(), ang.data(), az.data(),
                     opt, params, out.data(), passes);
  MF_GUARD_END
}

MF_API int mf_group_z0(mf_group* g, float* z0) {
  if (!g || !z0) return set_error(MF_ERR_ARG, "null argument");
  memcpy(z0, g->z0.data(), sizeof(float) * g->B);
  return MF_OK;
}

}  // extern "C"
