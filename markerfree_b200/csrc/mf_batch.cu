// Projection matching of many series in lockstep (a "group").
//
// Reference: Markerfree/src/method/ProjAlign.cpp:48-179 (Setup, DoIt, DoItBin) and
// Markerfree/src/main/Process.cpp:272-319 (mProjAlign, ProjAlignOnce), which align
// one series at a time.  Within a pass the held-out tilts of one series are
// sequential, so one series cannot fill a B200; series, however, are
// independent.  A group takes up to kMaxGroup series of the same shape and
// precision and runs the i-th held-out tilt of every series together: each stage
// of the pass (correction, R-weight FFTs, re-projection, normalisation,
// cross-correlation FFTs, filter, peak and parameter update, re-correction) is
// one launch over the whole group.  A per-series `active` flag in device memory
// lets the same launches serve every iteration of ProjAlignOnce even though each
// series leaves that loop after its own number of passes (the pass can also be
// captured once into a CUDA graph; `use_graph` below says why it is not by
// default).  Results per series are the same as when the series is
// aligned alone: the per-series arithmetic and its order are unchanged.
#include <algorithm>
#include <cstring>

#include "mf_series.hpp"
#include "mf_xcorr.hpp"

using namespace mf;

struct mf_group {
  mf_context* ctx = nullptr;
  std::vector<mf_series*> ser;
  int B = 0, nx = 0, ny = 0, nz = 0, n = 0;
  int bin = 1, xb = 0, yb = 0, pad = 0, cmp = 0, thick = 0, nproj = 10, prec = MF_PREC_FP32;
  int ytiles = 0, xpitch = 0, tc_nb = 256;
  size_t bpix = 0, ppix = 0;
  std::vector<std::vector<int>> order;
  std::vector<int> active;
  std::vector<float> z0;
  // device tables
  DevBuf d_ser, d_steps, d_active, d_order, d_bp, d_normptr, d_applyjobs, d_tiltidx;
  DevBuf d_maxerr, d_z0, d_err, d_meas, d_tcerr;
  // device buffers (series-major, contiguous over the group)
  DevBuf corr, scratch, corr16, tflags, rowflags, reproj, cc, recorr, recorr_out;
  DevBuf mpart, stats, ppart, mask;
  ReprojOpSet ops;
  TcOpSet tcops;
  TmaDesc imgmap;
  std::vector<TcJob> tcjobs;  // [n][B]
  cufftHandle rows_fwd_all = 0, rows_inv_all = 0, rows_fwd_one = 0, rows_inv_one = 0;
  cufftHandle cc_fwd = 0, cc_inv = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_kernels = 0;
  // Group passes launch eagerly: capturing and instantiating the graph of a group
  // pass (thousands of nodes, 8 series) cost more than its six replays saved
  // (bench step 2058 ms with the graph, 1564 ms without).
  bool use_graph = false;
  std::vector<cudaEvent_t> events;  // 3 per step when the context profiles
  double op_bytes = 0, op_fma = 0;  // mean compulsory bytes / MACs of one operator apply
  ~mf_group() {
    if (graph) cudaGraphExecDestroy(graph);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
};

namespace mf {

// corr[b][ip_b] = recorr_out[b] for the active series of a step
__global__ void k_group_scatter(const float* __restrict__ src, const GroupSeriesDev* __restrict__ ser,
                                const GroupStepDev* __restrict__ steps,
                                const int* __restrict__ active, size_t bpix) {
  const int b = blockIdx.y;
  if (active[b] == 0) return;
  const float4* s = reinterpret_cast<const float4*>(src + (size_t)b * bpix);
  float4* d = reinterpret_cast<float4*>(ser[b].corr + (size_t)steps[b].ip * bpix);
  const size_t n4 = bpix / 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x)
    d[i] = s[i];
}

static int group_setup(mf_group* g, float zshift, int align_z, int nproj) {
  StageTimer timer(&g->ctx->c, kStageSetup);
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B, nx = g->nx, ny = g->ny, nz = g->nz;
  int bx = (int)((float)nx / 2048.0f + 0.5f), by = (int)((float)ny / 2048.0f + 0.5f);
  g->bin = std::max(1, std::max(bx, by));
  g->xb = nx / g->bin / 2 * 2;
  g->yb = ny / g->bin / 2 * 2;
  g->pad = (g->xb / 2 + 1) * 2;
  g->cmp = g->pad / 2;
  g->thick = align_z / g->bin / 2 * 2;
  g->nproj = nproj;
  if (nproj <= 0) return set_error(MF_ERR_ARG, "nproj must be > 0");
  if (g->thick < 2) return set_error(MF_ERR_ARG, "slab thickness %d too small", g->thick);
  const int xb = g->xb, yb = g->yb, pad = g->pad;
  g->bpix = (size_t)xb * yb;
  g->ppix = (size_t)pad * yb;
  g->ytiles = (yb + kApplyTileY - 1) / kApplyTileY;
  g->n = nz - 1;
  const int n = g->n;
  // geometry of every series: outward order and neighbour ranges (ProjAlign.cpp:151-176)
  std::vector<ReprojGeom> geoms;
  std::vector<GroupStepDev> steps((size_t)n * B);
  std::vector<float> bp;
  std::vector<int> orders;
  std::vector<int> zts(B);
  g->order.assign(B, {});
  for (int b = 0; b < B; ++b) {
    mf_series* s = g->ser[b];
    const int zt = frame_idx_from_tilt(nz, s->angles.data(), 0.0f);
    zts[b] = zt;
    std::vector<unsigned char> skip(nz, 1);
    skip[zt] = 0;
    std::vector<ReprojGeom> gb;
    for (int i = 1; i < nz; ++i) {
      for (int side = 0; side < 2; ++side) {
        int ip = side == 0 ? zt + i : zt - i;
        if (ip < 0 || ip >= nz) continue;
        int rg[2];
        find_proj_range(s->angles.data(), nz, skip.data(), ip, nproj, rg);
        if (rg[0] < 0 || rg[1] < 0)
          return set_error(MF_ERR_GEOMETRY,
                           "series %d: no already-aligned tilt within 20.5 degrees of tilt %d "
                           "(%.2f)",
                           b, ip, s->angles[ip]);
        ReprojGeom gm;
        reproj_geometry(s->angles.data(), ip, rg[0], rg[1], xb, yb, g->thick, &gm);
        gb.push_back(gm);
        skip[ip] = 0;
      }
    }
    MF_TRY(fill_bp_device(c, s->angles.data(), &gb, st));
    for (const ReprojGeom& gm : gb) {
      const int k = (int)g->order[b].size();
      if (k >= n) break;
      GroupStepDev& sd = steps[(size_t)k * B + b];
      sd.ip = gm.ip;
      sd.i0 = gm.i0;
      sd.nk = gm.nk;
      sd.ray_len = gm.ray_len;
      sd.thick = gm.thick;
      sd.bp_off = (int)bp.size();
      sd.fcos = gm.fcos;
      sd.fsin = gm.fsin;
      bp.insert(bp.end(), gm.bp.begin(), gm.bp.end());
      g->order[b].push_back(gm.ip);
      geoms.push_back(gm);
    }
    if ((int)g->order[b].size() != n)
      return set_error(MF_ERR_GEOMETRY, "series %d: %d held-out tilts instead of %d", b,
                       (int)g->order[b].size(), n);
    orders.insert(orders.end(), g->order[b].begin(), g->order[b].end());
  }
  // buffers
  MF_TRY(g->corr.alloc(sizeof(float) * g->bpix * nz * B));
  MF_TRY(g->scratch.alloc(sizeof(float) * g->ppix * nz * B));
  MF_TRY(g->reproj.alloc(sizeof(float) * g->bpix * B));
  MF_TRY(g->cc.alloc(sizeof(float) * g->ppix * 2 * B));
  MF_TRY(g->recorr.alloc(sizeof(float) * g->ppix * B));
  MF_TRY(g->recorr_out.alloc(sizeof(float) * g->bpix * B));
  MF_TRY(g->mpart.alloc(sizeof(double2) * moment_parts(yb) * 2 * B));
  MF_TRY(g->stats.alloc(sizeof(float2) * 2 * B));
  MF_TRY(g->mask.alloc(sizeof(float) * g->bpix));
  MF_TRY(make_round_mask(c, xb, yb, (float)((pad / 2 - 1) * 2) * 0.5f, (float)yb * 0.5f,
                         (float)pad, (float)yb, 4.0f, g->mask.as<float>(), st));
  MF_TRY(g->ppart.alloc(sizeof(float2) * kPeakParts * B));
  MF_TRY(g->rowflags.alloc(sizeof(int) * g->ytiles * B));
  MF_TRY(g->d_steps.alloc(sizeof(GroupStepDev) * steps.size()));
  MF_TRY(g->d_order.alloc(sizeof(int) * std::max<size_t>(orders.size(), 1)));
  MF_TRY(g->d_bp.alloc(sizeof(float) * std::max<size_t>(bp.size(), 1)));
  MF_TRY(g->d_active.alloc(sizeof(int) * B));
  MF_TRY(g->d_maxerr.alloc(sizeof(float) * B));
  MF_TRY(g->d_z0.alloc(sizeof(float) * B));
  MF_TRY(g->d_err.alloc(sizeof(float) * nz * B));
  MF_TRY(g->d_meas.alloc(sizeof(float) * 2 * nz * B));
  MF_TRY(g->d_tcerr.alloc(sizeof(int)));
  MF_TRY(g->d_ser.alloc(sizeof(GroupSeriesDev) * B));
  MF_TRY(g->d_normptr.alloc(sizeof(float*) * 2 * B * (size_t)n));
  MF_TRY(g->d_tiltidx.alloc(sizeof(int) * B * (size_t)n));
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
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_err.p, 0, sizeof(float) * nz * B, st));
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_meas.p, 0, sizeof(float) * 2 * nz * B, st));
  MF_CHECK_CUDA(cudaMemsetAsync(g->d_tcerr.p, 0, sizeof(int), st));
  std::vector<GroupSeriesDev> sd(B);
  std::vector<const float*> normptr((size_t)2 * B * n);
  std::vector<int> tiltidx((size_t)B * n);
  float* corr = g->corr.as<float>();
  for (int b = 0; b < B; ++b) {
    mf_series* s = g->ser[b];
    GroupSeriesDev& d = sd[b];
    d.stack = s->stack.as<float>();
    d.stack_t = s->stack_t.as<float>();
    d.sx = s->d_sx.as<float>();
    d.sy = s->d_sy.as<float>();
    d.sx64 = s->dev_sx64();
    d.sy64 = s->dev_sy64();
    d.rot = s->d_rot.as<float>();
    d.angles = s->d_angles.as<float>();
    d.z0 = g->d_z0.as<float>() + b;
    d.err = g->d_err.as<float>() + (size_t)b * nz;
    d.meas = g->d_meas.as<float>() + (size_t)b * 2 * nz;
    d.corr = corr + (size_t)b * nz * g->bpix;
    d.order = g->d_order.as<int>() + (size_t)b * n;
    d.zt = zts[b];
    d.pad0 = 0;
    for (int k = 0; k < n; ++k) {
      const int ip = g->order[b][k];
      normptr[(size_t)k * 2 * B + 2 * b] = g->reproj.as<float>() + (size_t)b * g->bpix;
      normptr[(size_t)k * 2 * B + 2 * b + 1] = d.corr + (size_t)ip * g->bpix;
      tiltidx[(size_t)k * B + b] = b * nz + ip;
    }
  }
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_ser.p, sd.data(), sizeof(GroupSeriesDev) * B,
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_normptr.p, normptr.data(), sizeof(float*) * normptr.size(),
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_tiltidx.p, tiltidx.data(), sizeof(int) * tiltidx.size(),
                                cudaMemcpyHostToDevice, st));
  // re-projection operators of every (series, step): geometry index b * n + k
  if (g->prec != MF_PREC_FP32) {
    g->xpitch = (xb + 7) / 8 * 8;
    MF_TRY(g->corr16.alloc((size_t)2 * g->xpitch * yb * nz * B));
    MF_TRY(g->tflags.alloc(sizeof(int) * (size_t)nz * B * g->ytiles * kFlagParts));
    MF_TRY(build_reproj_tc_ops(c, geoms, g->prec, &g->tcops, st));
    g->tcjobs.resize((size_t)n * B);
    for (int b = 0; b < B; ++b)
      for (int k = 0; k < n; ++k) {
        const TcOpView& v = g->tcops.ops[(size_t)b * n + k];
        g->tcjobs[(size_t)k * B + b] =
            TcJob{v.xt, v.colvalid, g->reproj.as<float>() + (size_t)b * g->bpix, b * nz, 0};
      }
    // tile rows: timed on the first step of this group's shape, on a zeroed
    // 16-bit stack (the launches only write the re-projection buffers, which
    // every pass overwrites)
    MF_CHECK_CUDA(cudaMemsetAsync(g->corr16.p, 0, g->corr16.bytes, st));
    MF_TRY(tc_autotune_rows(
        c, xb, yb, B, g->prec,
        [&](int nb) -> int {
          TmaDesc m;
          MF_TRY(tc_image_map(g->corr16.p, g->prec, xb, g->xpitch, yb, nz * B, nb, &m));
          return launch_reproject_tc_group(c, g->tcops, g->tcjobs.data(), B, nullptr, xb, yb, m,
                                           nb, g->d_tcerr.as<int>(), st);
        },
        g->d_tcerr.as<int>(), &g->tc_nb, st));
    MF_TRY(tc_prepare(c, g->tc_nb));
    MF_TRY(tc_image_map(g->corr16.p, g->prec, xb, g->xpitch, yb, nz * B, g->tc_nb, &g->imgmap));
    MF_CHECK_CUDA(cudaMemsetAsync(g->d_tcerr.p, 0, sizeof(int), st));
  } else {
    MF_TRY(build_reproj_ops(c, geoms, &g->ops, st));
    std::vector<ApplyJob> jobs((size_t)n * B);
    for (int b = 0; b < B; ++b)
      for (int k = 0; k < n; ++k) {
        const ReprojOpView& v = g->ops.ops[(size_t)b * n + k];
        jobs[(size_t)k * B + b] =
            ApplyJob{v.tiles, v.colvalid, sd[b].corr, g->reproj.as<float>() + (size_t)b * g->bpix,
                     g->rowflags.as<int>() + (size_t)b * g->ytiles};
      }
    MF_TRY(g->d_applyjobs.alloc(sizeof(ApplyJob) * jobs.size()));
    MF_CHECK_CUDA(cudaMemcpyAsync(g->d_applyjobs.p, jobs.data(), sizeof(ApplyJob) * jobs.size(),
                                  cudaMemcpyHostToDevice, st));
  }
  const double nops = (double)B * n;
  g->op_bytes = (g->prec != MF_PREC_FP32 ? g->tcops.bytes : g->ops.bytes) / nops;
  g->op_fma = (g->prec != MF_PREC_FP32 ? g->tcops.fma : g->ops.fma) / nops;
  // FFT plans (cached per context)
  mf_context* ctx = g->ctx;
  // The same plan shapes as a single series' pass, executed once per series: a
  // plan batched over the group may round differently, and a different rounding
  // can flip a near-tied decision later (tilt-axis candidates, nearest-neighbour
  // re-correction), so per-series execution keeps each result identical to the
  // series aligned alone.
  MF_TRY(ctx->plan({0, xb, yb, (long long)nz * yb}, &g->rows_fwd_all));
  MF_TRY(ctx->plan({1, xb, yb, (long long)nz * yb}, &g->rows_inv_all));
  MF_TRY(ctx->plan({0, xb, yb, (long long)yb}, &g->rows_fwd_one));
  MF_TRY(ctx->plan({1, xb, yb, (long long)yb}, &g->rows_inv_one));
  MF_TRY(ctx->plan({2, xb, yb, 2}, &g->cc_fwd));
  MF_TRY(ctx->plan({3, xb, yb, 1}, &g->cc_inv));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// One projection-matching pass over the active series (the group form of
// pa_enqueue in mf_series.cu).
static int group_enqueue(mf_group* g) {
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B, nz = g->nz, n = g->n, xb = g->xb, yb = g->yb, pad = g->pad, cmp = g->cmp;
  const size_t bpix = g->bpix, ppix = g->ppix;
  const bool tc = g->prec != MF_PREC_FP32;
  const GroupSeriesDev* ser = g->d_ser.as<GroupSeriesDev>();
  const GroupStepDev* steps = g->d_steps.as<GroupStepDev>();
  const int* active = g->d_active.as<int>();
  float* corr = g->corr.as<float>();
  float* scratch = g->scratch.as<float>();
  float* cc = g->cc.as<float>();
  if (!tc) MF_CHECK_CUDA(cudaMemsetAsync(g->rowflags.p, 0, sizeof(int) * g->ytiles * B, st));
  // CorrTomoStack::DoIt for every tilt of every active series
  GroupCorrArgs ca{ser, nullptr, active, g->nx, g->ny, nz, g->bin, 1, scratch, pad, ppix};
  MF_TRY(launch_correct_group(c, ca, B * nz, st));
  for (int b = 0; b < B; ++b) {
    float* sb = scratch + (size_t)b * nz * ppix;
    MF_CHECK_CUFFT(cufftExecR2C(g->rows_fwd_all, sb, (cufftComplex*)sb));
  }
  MF_TRY(launch_rweight(c, (cufftComplex*)scratch, cmp, B * nz * yb, st));
  for (int b = 0; b < B; ++b)
    MF_CHECK_CUFFT(cufftExecC2R(g->rows_inv_all, (cufftComplex*)(scratch + (size_t)b * nz * ppix),
                                corr + (size_t)b * nz * bpix));
  if (tc)
    MF_TRY(launch_to_half(c, corr, xb, yb, nullptr, 0, B * nz, g->prec, g->corr16.p, g->xpitch,
                          g->tflags.as<int>(), st));
  MF_TRY(fit_z0_group(c, ser, active, B, nz, st));
  const float mcx = (float)((pad / 2 - 1) * 2) * 0.5f, mcy = (float)yb * 0.5f;
  const bool prof = c->profiling && (int)g->events.size() >= 3 * n;
  for (int k = 0; k < n; ++k) {
    const GroupStepDev* sk = steps + (size_t)k * B;
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k], st));
    if (tc) {
      MF_TRY(launch_reproject_tc_group(c, g->tcops, g->tcjobs.data() + (size_t)k * B, B, active,
                                       xb, yb, g->imgmap, g->tc_nb, g->d_tcerr.as<int>(), st));
      MF_TRY(launch_reproject_exact_group(c, ser, sk, active, B, nz, xb, yb, g->d_bp.as<float>(),
                                          g->tflags.as<int>(), nullptr, g->reproj.as<float>(),
                                          st));
    } else {
      const int ntiles = (xb + kOpTileX - 1) / kOpTileX;
      MF_TRY(launch_reproject_apply_group(c, g->ops, g->d_applyjobs.as<ApplyJob>() + (size_t)k * B,
                                          active, B, xb, yb, ntiles, st));
      MF_TRY(launch_reproject_exact_group(c, ser, sk, active, B, nz, xb, yb, g->d_bp.as<float>(),
                                          nullptr, g->rowflags.as<int>(), g->reproj.as<float>(),
                                          st));
    }
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k + 1], st));
    // MeaAlignProj for every series: PANorm both images, FFT, filter, inverse, peak
    MF_TRY(norm_mask_pad_group(c, g->d_normptr.as<const float*>() + (size_t)k * 2 * B, active,
                               2 * B, xb, yb, pad, ppix, mcx, mcy, (float)pad, (float)yb, 4.0f,
                               g->mask.as<float>(), cc, g->mpart.as<double2>(),
                               g->stats.as<float2>(), st));
    for (int b = 0; b < B; ++b) {
      float* cb = cc + (size_t)b * 2 * ppix;
      MF_CHECK_CUFFT(cufftExecR2C(g->cc_fwd, cb, (cufftComplex*)cb));
    }
    MF_TRY(xcorr_filter(c, (cufftComplex*)cc, ppix, nullptr, (cufftComplex*)(cc + ppix), ppix, B,
                        cmp, yb, 500.0f, 1.0f, st));
    for (int b = 0; b < B; ++b) {
      float* mb = cc + (size_t)(2 * b + 1) * ppix;
      MF_CHECK_CUFFT(cufftExecC2R(g->cc_inv, (cufftComplex*)mb, mb));
    }
    MF_TRY(pa_peak_update_group(c, cc + ppix, 2 * ppix, pad, xb, yb, g->ppart.as<float2>(), ser,
                                sk, active, B, g->nx, g->ny, st));
    // re-correct the aligned tilt of every series (mCorrectProj)
    GroupCorrArgs rc{ser, sk, active, g->nx, g->ny, nz, g->bin, 1, g->recorr.as<float>(), pad,
                     ppix};
    MF_TRY(launch_correct_group(c, rc, B, st));
    for (int b = 0; b < B; ++b) {
      float* rb = g->recorr.as<float>() + (size_t)b * ppix;
      MF_CHECK_CUFFT(cufftExecR2C(g->rows_fwd_one, rb, (cufftComplex*)rb));
    }
    MF_TRY(launch_rweight(c, (cufftComplex*)g->recorr.as<float>(), cmp, B * yb, st));
    for (int b = 0; b < B; ++b)
      MF_CHECK_CUFFT(cufftExecC2R(g->rows_inv_one,
                                  (cufftComplex*)(g->recorr.as<float>() + (size_t)b * ppix),
                                  g->recorr_out.as<float>() + (size_t)b * bpix));
    k_group_scatter<<<dim3(64, B), 256, 0, st>>>(g->recorr_out.as<float>(), ser, sk, active, bpix);
    c->launches++;
    MF_CHECK_CUDA(cudaGetLastError());
    if (tc)
      MF_TRY(launch_to_half(c, corr, xb, yb, g->d_tiltidx.as<int>() + (size_t)k * B, 0, B, g->prec,
                            g->corr16.p, g->xpitch, g->tflags.as<int>(), st));
    if (prof) MF_CHECK_CUDA(cudaEventRecord(g->events[3 * k + 2], st));
  }
  MF_TRY(max_err_group(c, ser, active, B, n, g->d_maxerr.as<float>(), st));
  return MF_OK;
}

// One pass over the series with active[b] != 0; max_err[b] receives each active
// series' largest measured shift (inactive entries are left as they are).
static int group_doit(mf_group* g, const int* active, float* max_err) {
  StageTimer timer(&g->ctx->c, kStagePass);
  Context* c = &g->ctx->c;
  cudaStream_t st = c->stream;
  const int B = g->B;
  g->active.assign(active, active + B);
  for (int b = 0; b < B; ++b) MF_TRY(g->ser[b]->upload_params());
  MF_CHECK_CUDA(cudaMemcpyAsync(g->d_active.p, g->active.data(), sizeof(int) * B,
                                cudaMemcpyHostToDevice, st));
  // Profiled passes run eagerly: events recorded by graph nodes cannot be timed.
  while (c->profiling && (int)g->events.size() < 3 * g->n) {
    cudaEvent_t e;
    MF_CHECK_CUDA(cudaEventCreate(&e));
    g->events.push_back(e);
  }
  if (g->use_graph && !g->graph && !c->profiling) {
    int64_t l0 = c->launches;
    cudaGraph_t gr = nullptr;
    std::unique_lock<std::recursive_mutex> fft_lock(fft_mutex());
    MF_CHECK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = group_enqueue(g);
    cudaError_t ec = cudaStreamEndCapture(st, &gr);
    fft_lock.unlock();
    g->graph_kernels = c->launches - l0;
    c->launches = l0;
    if (rc != MF_OK || ec != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      cudaGetLastError();
      g->use_graph = false;
    } else {
      cudaError_t ei = cudaGraphInstantiate(&g->graph, gr, 0);
      cudaGraphDestroy(gr);
      if (ei != cudaSuccess) {
        cudaGetLastError();
        g->graph = nullptr;
        g->use_graph = false;
      }
    }
  }
  if (g->graph && !c->profiling) {
    MF_CHECK_CUDA(cudaGraphLaunch(g->graph, st));
    c->launches += g->graph_kernels;
  } else {
    MF_TRY(group_enqueue(g));
  }
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
  int nact = 0;
  for (int b = 0; b < B; ++b)
    if (active[b]) {
      max_err[b] = me[b];
      g->ser[b]->pa.z0 = g->z0[b];
      nact++;
    }
  if (c->profiling && (int)g->events.size() >= 3 * g->n) {
    // stage times of this pass: [0] re-projection launches (one per step for the
    // whole group), [2] the rest of each step; bytes and MACs of the active series
    for (int k = 0; k < g->n; ++k) {
      float a = 0.0f, b2 = 0.0f;
      MF_CHECK_CUDA(cudaEventElapsedTime(&a, g->events[3 * k], g->events[3 * k + 1]));
      MF_CHECK_CUDA(cudaEventElapsedTime(&b2, g->events[3 * k + 1], g->events[3 * k + 2]));
      c->stage[0] += a;
      c->stage[2] += b2;
    }
    c->stage[1] += g->n;
    c->stage[3] += 1;
    c->stage[4] += g->op_bytes * g->n * nact;
    c->stage[5] += g->op_fma * g->n * nact;
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

int group_create(mf_context* ctx, mf_series* const* series, int nser, float zshift, int align_z,
                 int nproj, mf_group** out) {
  if (!out) return set_error(MF_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (!ctx || !series || nser < 1 || nser > kMaxGroup)
    return set_error(MF_ERR_ARG, "a group holds 1..%d series (got %d)", kMaxGroup, nser);
  for (int b = 0; b < nser; ++b) {
    const mf_series* s = series[b];
    if (!s) return set_error(MF_ERR_ARG, "null series %d", b);
    if (s->ctx != ctx) return set_error(MF_ERR_ARG, "series %d belongs to another context", b);
    if (s->gpu != ctx->c.gpu) return set_error(MF_ERR_ARG, "series %d is on another GPU", b);
    if (s->nx != series[0]->nx || s->ny != series[0]->ny || s->nz != series[0]->nz ||
        s->precision != series[0]->precision)
      return set_error(MF_ERR_ARG,
                       "series %d differs in shape or precision from series 0 (%d x %d x %d)", b,
                       series[0]->nx, series[0]->ny, series[0]->nz);
  }
  mf_group* g = new mf_group();
  g->ctx = ctx;
  g->ser.assign(series, series + nser);
  g->B = nser;
  g->nx = series[0]->nx;
  g->ny = series[0]->ny;
  g->nz = series[0]->nz;
  g->prec = series[0]->precision;
  int rc = group_setup(g, zshift, align_z, nproj);
  if (rc != MF_OK) {
    delete g;
    return rc;
  }
  *out = g;
  return MF_OK;
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

// Process::DoIt minus file I/O (Process.cpp:34-92) for n series of one shape:
// every series is uploaded and pre-processed, coarse-aligned stage by stage with
// the others of its group of up to kMaxGroup, projection-matched with them in
// lockstep, then corrected into d_out[i].
MF_API int mf_align_many_device(mf_context* ctx, int n, const float* const* d_raw, int nx, int ny,
                                int nz, const float* const* file_angles, const mf_options* opt,
                                mf_align_param* params, float* const* d_out, int* passes) {
  MF_GUARD_BEGIN
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
    rc = mf_series_create_device(ctx, d_raw[i], nx, ny, nz, file_angles[i], &ser[i]);
    if (rc == MF_OK) ser[i]->precision = (mf_precision)opt->precision;
  }
  // the coarse stages stage by stage over groups of series (one host wait per stage)
  for (int g0 = 0; g0 < n && rc == MF_OK && opt->align_z != 0; g0 += kMaxGroup)
    rc = coarse_align_many(ser.data() + g0, std::min(kMaxGroup, n - g0), opt->pitch_angle,
                           opt->offset);
  for (int g0 = 0; g0 < n && rc == MF_OK && opt->align_z != 0; g0 += kMaxGroup) {
    const int m = std::min(kMaxGroup, n - g0);
    mf_group* g = nullptr;
    rc = group_create(ctx, ser.data() + g0, m, opt->zshift, opt->align_z, opt->nproj, &g);
    if (rc == MF_OK) rc = group_proj_align(g, passes ? passes + g0 : nullptr);
    delete g;
  }
  if (opt->align_z == 0 && passes)
    for (int i = 0; i < n; ++i) passes[i] = 0;
  for (int i = 0; i < n && rc == MF_OK; ++i) {
    if (d_out && d_out[i]) rc = correct_stack_device(ser[i], opt->out_bin, d_out[i]);
    if (rc == MF_OK) rc = mf_series_get_param(ser[i], &params[i]);
  }
  if (rc == MF_OK && cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
    rc = set_error(MF_ERR_CUDA, "stream synchronize failed");
  cleanup();
  return rc;
  MF_GUARD_END
}

MF_API int mf_group_z0(mf_group* g, float* z0) {
  if (!g || !z0) return set_error(MF_ERR_ARG, "null argument");
  memcpy(z0, g->z0.data(), sizeof(float) * g->B);
  return MF_OK;
}

}  // extern "C"
