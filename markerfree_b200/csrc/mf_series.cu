// Alignment stages on a device-resident series.
//
// Reference: Markerfree/src/main/Process.cpp (pipeline and schedule),
// Markerfree/src/method/ProjAlign.cpp (projection matching), Transform.cpp and
// FindOffset.cu (coarse stages), Rotate.cu (tilt axis), CorrStack.cu (correction).
// The reference re-reads every slice from a scratch MRC on disk for every
// correction and drives the GPU with one synchronous call per image row.  Here
// the pre-processed stack stays in HBM, a projection-matching pass is a fixed
// sequence of kernels and cuFFT calls captured once into a CUDA graph, and only
// the pass's largest shift, the rotation-centre z and the shifts come back to
// the host after each pass.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "mf_series.hpp"
#include "mf_xcorr.hpp"

using namespace mf;

// Every cuFFT call of the process (planning, execution, destruction) and every
// stream capture (which records cuFFT launches) holds one lock: plans created
// while other threads (the serving workers) planned, executed or captured
// crashed inside cuFFT's planner.  Executions are asynchronous launches, so the
// lock is held for microseconds.
std::recursive_mutex& mf::fft_mutex() {
  static std::recursive_mutex m;
  return m;
}

mf_context::~mf_context() {
  std::lock_guard<std::recursive_mutex> lk(fft_mutex());
  for (auto& kv : plans) cufftDestroy(kv.second);
  plans.clear();
  for (int i = 0; i <= kFftStreams; ++i)
    if (work[i]) cudaFree(work[i]);
  for (void* p : retired_work) cudaFree(p);
  for (int i = 0; i < kFftStreams; ++i) {
    if (aux[i]) cudaStreamDestroy(aux[i]);
    if (join_ev[i]) cudaEventDestroy(join_ev[i]);
  }
  if (fork_ev) cudaEventDestroy(fork_ev);
  if (c.stream) cudaStreamDestroy(c.stream);
}

int mf_context::ensure_aux() {
  if (fork_ev) return MF_OK;
  for (int i = 0; i < kFftStreams; ++i) {
    MF_CHECK_CUDA(cudaStreamCreateWithFlags(&aux[i], cudaStreamNonBlocking));
    MF_CHECK_CUDA(cudaEventCreateWithFlags(&join_ev[i], cudaEventDisableTiming));
  }
  MF_CHECK_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  return MF_OK;
}

int mf_context::plan(const std::vector<long long>& key, cufftHandle* out) {
  auto it = plans.find(key);
  if (it != plans.end()) {
    *out = it->second;
    return MF_OK;
  }
  // key: kind (0 rows R2C in place, 1 rows C2R out of place, 2 2-D R2C in place,
  //            3 2-D C2R in place, 4 1-D R2C lines, 5 2-D C2R pairs), nx, ny, batch,
  //      and optionally the side stream the plan is bound to
  std::lock_guard<std::recursive_mutex> lk(fft_mutex());
  const int slot = (key.size() > 4 && key[4] >= 0) ? (int)key[4] : kFftStreams;
  if (slot > kFftStreams) return set_error(MF_ERR_ARG, "FFT side stream %d out of range", slot);
  if (slot < kFftStreams) MF_TRY(ensure_aux());
  cudaStream_t bind = slot < kFftStreams ? aux[slot] : c.stream;
  long long kind = key[0];
  int nx = (int)key[1], ny = (int)key[2], batch = (int)key[3];
  int pad = (nx / 2 + 1) * 2, cmp = nx / 2 + 1;
  cufftHandle h;
  if (cufftCreate(&h) != CUFFT_SUCCESS) return set_error(MF_ERR_CUFFT, "cufftCreate failed");
  // The work area is the context's, one per stream (see work[]): plans of one
  // stream run one after another, so they share it.
  cufftSetAutoAllocation(h, 0);
  size_t ws = 0;
  cufftResult r;
  if (kind == 0) {
    int n[1] = {nx}, inem[1] = {pad}, onem[1] = {cmp};
    r = cufftMakePlanMany(h, 1, n, inem, 1, pad, onem, 1, cmp, CUFFT_R2C, batch, &ws);
  } else if (kind == 1) {
    int n[1] = {nx}, inem[1] = {cmp}, onem[1] = {nx};
    r = cufftMakePlanMany(h, 1, n, inem, 1, cmp, onem, 1, nx, CUFFT_C2R, batch, &ws);
  } else if (kind == 4) {
    // 1-D R2C in place with the default padded layout (tilt-axis lines)
    r = cufftMakePlan1d(h, nx, CUFFT_R2C, batch, &ws);
  } else if (kind == 5) {
    // 2-D C2R in place over `batch` maps spaced two padded images apart
    int n[2] = {ny, nx}, inem[2] = {ny, cmp}, onem[2] = {ny, pad};
    r = cufftMakePlanMany(h, 2, n, inem, 1, 2 * ny * cmp, onem, 1, 2 * ny * pad, CUFFT_C2R,
                          batch, &ws);
  } else if (kind == 2) {
    int n[2] = {ny, nx}, inem[2] = {ny, pad}, onem[2] = {ny, cmp};
    r = cufftMakePlanMany(h, 2, n, inem, 1, ny * pad, onem, 1, ny * cmp, CUFFT_R2C, batch, &ws);
  } else {
    int n[2] = {ny, nx}, inem[2] = {ny, cmp}, onem[2] = {ny, pad};
    r = cufftMakePlanMany(h, 2, n, inem, 1, ny * cmp, onem, 1, ny * pad, CUFFT_C2R, batch, &ws);
  }
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    return set_error(r == CUFFT_ALLOC_FAILED ? MF_ERR_NOMEM : MF_ERR_CUFFT,
                     "cufftMakePlanMany(kind %lld, %d x %d, batch %d) failed: %d", kind, nx, ny,
                     batch, (int)r);
  }
  if (ws > work_bytes[slot]) {
    // grow this stream's work area and point every plan of the stream at the new
    // one.  The old area is kept until the context goes: a pass captured into a
    // CUDA graph holds the address its plans had at capture time.
    void* p = nullptr;
    if (cudaMalloc(&p, ws) != cudaSuccess) {
      cudaGetLastError();
      cufftDestroy(h);
      return set_error(MF_ERR_NOMEM, "FFT work area of %zu MB: device memory exhausted",
                       ws >> 20);
    }
    if (work[slot]) retired_work.push_back(work[slot]);
    work[slot] = p;
    work_bytes[slot] = ws;
    for (auto& kv : plans) {
      const int ks = (kv.first.size() > 4 && kv.first[4] >= 0) ? (int)kv.first[4] : kFftStreams;
      if (ks == slot) cufftSetWorkArea(kv.second, work[slot]);
    }
  }
  if (ws > 0) cufftSetWorkArea(h, work[slot]);
  cufftSetStream(h, bind);
  plans[key] = h;
  *out = h;
  return MF_OK;
}

namespace mf {

ProjAlignState::~ProjAlignState() {
  if (graph) cudaGraphExecDestroy(graph);
  graph = nullptr;
  for (cudaEvent_t e : events) cudaEventDestroy(e);
  events.clear();
}

// ---------------------------------------------------------------------------
__global__ void k_pad_copy(const float* __restrict__ src, int w, int h, int pad,
                           float* __restrict__ dst) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  int z = blockIdx.z;
  if (x >= pad || y >= h) return;
  dst[((size_t)z * h + y) * pad + x] = (x < w) ? src[((size_t)z * h + y) * w + x] : 0.0f;
}

int series_init(mf_series* s, mf_context* ctx, int nx, int ny, int nz, const float* file_angles) {
  s->ctx = ctx;
  s->gpu = ctx->c.gpu;
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  s->file_angles.assign(file_angles, file_angles + nz);
  s->angles = s->file_angles;
  if (nz > 1 && s->angles[0] > s->angles[1]) std::reverse(s->angles.begin(), s->angles.end());
  s->sx.assign(nz, 0.0f);
  s->sy.assign(nz, 0.0f);
  s->sx64.assign(nz, 0.0);
  s->sy64.assign(nz, 0.0);
  s->rot.assign(nz, 0.0f);
  s->angle_offset = 0.0f;
  MF_TRY(s->d_sx.alloc(sizeof(float) * nz));
  MF_TRY(s->d_sy.alloc(sizeof(float) * nz));
  MF_TRY(s->d_sx64.alloc(sizeof(double) * nz));
  MF_TRY(s->d_sy64.alloc(sizeof(double) * nz));
  MF_TRY(s->d_rot.alloc(sizeof(float) * nz));
  MF_TRY(s->d_angles.alloc(sizeof(float) * nz));
  return MF_OK;
}

}  // namespace mf

int mf_series::upload_params() {
  cudaStream_t st = ctx->c.stream;
  MF_CHECK_CUDA(cudaMemcpyAsync(d_sx.p, sx.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_sy.p, sy.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  if (shift64()) {
    for (int i = 0; i < nz; ++i) {
      if ((float)sx64[i] != sx[i]) sx64[i] = sx[i];
      if ((float)sy64[i] != sy[i]) sy64[i] = sy[i];
    }
    MF_CHECK_CUDA(cudaMemcpyAsync(d_sx64.p, sx64.data(), sizeof(double) * nz,
                                  cudaMemcpyHostToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(d_sy64.p, sy64.data(), sizeof(double) * nz,
                                  cudaMemcpyHostToDevice, st));
  }
  MF_CHECK_CUDA(cudaMemcpyAsync(d_rot.p, rot.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_angles.p, angles.data(), sizeof(float) * nz,
                                cudaMemcpyHostToDevice, st));
  return MF_OK;
}

int mf_series::queue_download_shifts() {
  cudaStream_t st = ctx->c.stream;
  MF_CHECK_CUDA(cudaMemcpyAsync(sx.data(), d_sx.p, sizeof(float) * nz, cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(sy.data(), d_sy.p, sizeof(float) * nz, cudaMemcpyDeviceToHost, st));
  if (shift64()) {
    MF_CHECK_CUDA(cudaMemcpyAsync(sx64.data(), d_sx64.p, sizeof(double) * nz,
                                  cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(sy64.data(), d_sy64.p, sizeof(double) * nz,
                                  cudaMemcpyDeviceToHost, st));
  }
  return MF_OK;
}

int mf_series::download_shifts() {
  MF_TRY(queue_download_shifts());
  MF_CHECK_CUDA(cudaStreamSynchronize(ctx->c.stream));
  return MF_OK;
}

namespace mf {

// ---------------------------------------------------------------------------
// Transform::DoIt + Measure (Transform.cpp:60-97), all tilt pairs batched.  The
// pass is queued by transform_enqueue (its measured shifts land in page-locked
// slot `slot` of the context) and applied by transform_finish once the stream
// has been synchronised.
int transform_enqueue(mf_series* s, int slot, TransformJob* J) {
  Context* c = &s->ctx->c;
  cudaStream_t st = c->stream;
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  TransformState& T = s->tr;
  if (!T.ready) {
    int bx = (int)((float)nx / 1024.0f + 0.1f), by = (int)((float)ny / 1024.0f + 0.1f);
    T.bin = std::max(1, std::max(bx, by));
    T.xb = nx / T.bin / 2 * 2;
    T.yb = ny / T.bin / 2 * 2;
    T.pshx.assign(nz, 0.0f);
    T.pshy.assign(nz, 0.0f);
    T.ready = true;
  }
  const int xb = T.xb, yb = T.yb, pad = xb + 2, cmp = xb / 2 + 1;
  const size_t bpix = (size_t)xb * yb, ppix = (size_t)pad * yb;
  MF_TRY(s->upload_params());
  // device buffers are released stream-ordered on return, after the queued work
  DevBuf corr, pbuf, refs, imgs, part, stats, d_idx, d_refidx, d_mats, d_shifts, d_peakpart;
  MF_TRY(corr.alloc(sizeof(float) * bpix * nz));
  MF_TRY(pbuf.alloc(sizeof(float) * ppix * nz));
  MF_TRY(refs.alloc(sizeof(float) * ppix * nz));
  MF_TRY(launch_correct_bin(c, s->stack.as<float>(), s->stack_t.as<float>(),
                            nx, ny, nullptr, nz, s->d_sx.as<float>(),
                            s->d_sy.as<float>(), s->d_rot.as<float>(), 1, T.bin, 1,
                            corr.as<float>(), xb, bpix, st));
  k_pad_copy<<<dim3((pad + 63) / 64, (yb + 3) / 4, nz), dim3(64, 4), 0, st>>>(
      corr.as<float>(), xb, yb, pad, pbuf.as<float>());
  c->launches++;
  // pairs
  std::vector<int>& img_idx = J->img_idx;
  std::vector<int> ref_idx;
  std::vector<float> mats;
  img_idx.clear();
  for (int z = 0; z < nz; ++z) {
    int r = find_ref_index(nz, s->angles.data(), z);
    if (r == z) continue;
    img_idx.push_back(z);
    ref_idx.push_back(r);
    double ds = std::cos(kD2R * s->angles[r]) / std::cos(kD2R * s->angles[z]);
    float m[3];
    stretch_matrix((float)ds, s->rot[z], m);
    mats.insert(mats.end(), m, m + 3);
  }
  const int np = (int)img_idx.size();
  J->np = np;
  J->h_sh = nullptr;
  if (np == 0) return MF_OK;
  J->h_sh = (float2*)c->pinned.get(slot, sizeof(float2) * np);
  if (!J->h_sh) return MF_ERR_NOMEM;
  MF_TRY(imgs.alloc(sizeof(float) * ppix * np));
  MF_TRY(part.alloc(sizeof(double2) * moment_parts(yb) * std::max(nz, np)));
  MF_TRY(stats.alloc(sizeof(float2) * std::max(nz, np)));
  MF_TRY(d_idx.alloc(sizeof(int) * np));
  MF_TRY(d_refidx.alloc(sizeof(int) * np));
  MF_TRY(d_mats.alloc(sizeof(float) * 3 * np));
  MF_TRY(d_shifts.alloc(sizeof(float2) * np));
  MF_TRY(d_peakpart.alloc(sizeof(float2) * 32 * np));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_idx.p, img_idx.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_refidx.p, ref_idx.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_mats.p, mats.data(), sizeof(float) * 3 * np, cudaMemcpyHostToDevice, st));
  const float cx = xb * 0.5f, cy = yb * 0.5f, msx = xb * 1.0f, msy = yb * 1.0f;
  if (!T.mask.p) {  // one geometry for every stretch correlation of the series
    MF_TRY(T.mask.alloc(sizeof(float) * bpix));
    MF_TRY(make_round_mask(c, xb, yb, cx, cy, msx, msy, 4.0f, T.mask.as<float>(), st));
  }
  // references: normalise (mean, std) + round edge, all tilts
  MF_TRY(norm_mask_pad(c, pbuf.as<float>(), nullptr, pad, ppix, xb, yb, pad, ppix, nz, 1, cx, cy,
                       msx, msy, 4.0f, T.mask.as<float>(), refs.as<float>(), part.as<double2>(),
                       stats.as<float2>(), st));
  // images: stretch the padded raw copy, then normalise + round edge
  MF_TRY(stretch_many(c, pbuf.as<float>(), ppix, d_idx.as<int>(), xb, yb, pad, d_mats.as<float>(),
                      np, 1, imgs.as<float>(), ppix, st));
  MF_TRY(norm_mask_pad(c, imgs.as<float>(), nullptr, pad, ppix, xb, yb, pad, ppix, np, 1, cx, cy,
                       msx, msy, 4.0f, T.mask.as<float>(), imgs.as<float>(), part.as<double2>(),
                       stats.as<float2>(), st));
  cufftHandle fr, fi, inv;
  MF_TRY(s->ctx->plan({2, xb, yb, nz}, &fr));
  MF_TRY(s->ctx->plan({2, xb, yb, np}, &fi));
  MF_TRY(s->ctx->plan({3, xb, yb, np}, &inv));
  MF_CHECK_CUFFT(cufftExecR2C(fr, refs.as<cufftReal>(), refs.as<cufftComplex>()));
  MF_CHECK_CUFFT(cufftExecR2C(fi, imgs.as<cufftReal>(), imgs.as<cufftComplex>()));
  float scale = (float)(1.0 / ((cmp - 1) * 2) / yb);
  MF_TRY(xcorr_filter(c, refs.as<cufftComplex>(), ppix / 2, d_refidx.as<int>(),
                      imgs.as<cufftComplex>(), ppix / 2, np, cmp, yb, 400.0f, scale, st));
  MF_CHECK_CUFFT(cufftExecC2R(inv, imgs.as<cufftComplex>(), imgs.as<cufftReal>()));
  MF_TRY(cc_peaks(c, imgs.as<float>(), ppix, pad, xb, yb, np, d_peakpart.as<float2>(),
                  d_shifts.as<float2>(), st));
  MF_CHECK_CUDA(cudaMemcpyAsync(J->h_sh, d_shifts.p, sizeof(float2) * np, cudaMemcpyDeviceToHost,
                                st));
  return MF_OK;
}

int transform_finish(mf_series* s, TransformJob* J, float* max_err_out) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  TransformState& T = s->tr;
  const int xb = T.xb, yb = T.yb;
  float maxerr = 0.0f;
  float binx = nx * 1.0f / xb, biny = ny * 1.0f / yb;
  for (int p = 0; p < J->np; ++p) {
    int z = J->img_idx[p];
    T.pshx[z] = J->h_sh[p].x * binx;
    T.pshy[z] = J->h_sh[p].y * biny;
    float e = (float)std::sqrt(T.pshx[z] * T.pshx[z] + T.pshy[z] * T.pshy[z]);
    if (e > maxerr) maxerr = e;
  }
  // UpdateShift + UnStretch (Transform.cpp:99-157)
  int zt = frame_idx_from_tilt(nz, s->angles.data(), 0.0f);
  for (int i = 0; i < nz; ++i) {
    T.pshx[i] -= T.pshx[zt];
    T.pshy[i] -= T.pshy[zt];
  }
  auto unstretch = [&](int ref, int f, float* sum) {
    double ds = std::cos(s->angles[ref] * kD2R) / std::cos(s->angles[f] * kD2R);
    double d2t = 2 * kD2R * s->rot[f];
    double s2 = std::sin(d2t), c2 = std::cos(d2t);
    double P = 0.5 * (ds + 1), M = 0.5 * (ds - 1);
    float a0 = (float)(P + M * c2), a1 = (float)(1 * M * s2), a2 = (float)(P - M * c2);
    float det = a0 * a2 - a1 * a1;
    float m0 = a2 / det, m1 = -a1 / det, m2 = a0 / det;
    float buf = sum[0] * m0 + sum[1] * m1;
    sum[1] = sum[0] * m1 + sum[1] * m2;
    sum[0] = buf;
  };
  float sum[2] = {0.0f, 0.0f};
  for (int i = zt - 1; i >= 0; --i) {
    sum[0] += T.pshx[i];
    sum[1] += T.pshy[i];
    unstretch(i + 1, i, sum);
    s->sx[i] += sum[0];
    s->sy[i] += sum[1];
  }
  sum[0] = sum[1] = 0.0f;
  for (int i = zt + 1; i < nz; ++i) {
    sum[0] += T.pshx[i];
    sum[1] += T.pshy[i];
    unstretch(i - 1, i, sum);
    s->sx[i] += sum[0];
    s->sy[i] += sum[1];
  }
  if (max_err_out) *max_err_out = maxerr;
  return MF_OK;
}

int transform_doit(mf_series* s, float* max_err_out) {
  StageTimer timer(&s->ctx->c, kStageCoarse);
  TransformJob J;
  MF_TRY(transform_enqueue(s, 0, &J));
  MF_CHECK_CUDA(cudaStreamSynchronize(s->ctx->c.stream));
  return transform_finish(s, &J, max_err_out);
}

// ---------------------------------------------------------------------------
// CalcTIltAxis::DoIt + CLsetup (Rotate.cu:292-374): axis_enqueue queues one search
// (scores to the context's page-locked slot `slot`), axis_finish applies the
// arg-max rule once the stream has been synchronised.
int axis_enqueue(mf_series* s, float range, int num, int slot, AxisSearch* A) {
  if (num < 2) return set_error(MF_ERR_ARG, "tilt axis: need at least 2 candidates");
  Context* c = &s->ctx->c;
  const int nz = s->nz;
  int zt = frame_idx_from_tilt(nz, s->angles.data(), 0.0f);
  float axis0 = s->rot[zt];
  float step = range / (num - 1);
  std::vector<float>& cand = A->cand;
  cand.assign(num, 0.0f);
  cand[0] = axis0 - step * num / 2;
  for (int i = 1; i < num; ++i) cand[i] = cand[i - 1] + step;
  float fmin_size = 1e20f;
  for (int i = 0; i < num; ++i) {
    float fs = (float)std::fabs(std::sin(kD2R * cand[i]));
    float fc = (float)std::fabs(std::cos(kD2R * cand[i]));
    float s1 = (float)s->nx / (fs + 0.000001f);
    float s2 = (float)s->ny / (fc + 0.000001f);
    if (fmin_size > s1) fmin_size = s1;
    if (fmin_size > s2) fmin_size = s2;
  }
  int L = (int)fmin_size;
  L = L / 2 * 2 - 100;
  if (L < 4) return set_error(MF_ERR_ARG, "tilt axis: image too small (line length %d)", L);
  cufftHandle plan;
  MF_TRY(s->ctx->plan({4, L, 0, (long long)nz * num}, &plan));
  return tilt_axis_scores_enqueue(c, plan, s->stack.as<float>(), s->stack_t.as<float>(),
                                  s->d_neg.as<int>(), s->nx, s->ny, nz, s->angles.data(),
                                  s->sx.data(), s->sy.data(), zt, cand.data(), num, L, slot,
                                  &A->job, c->stream);
}

int axis_finish(mf_series* s, AxisSearch* A, float* axis_out, float* scores_out) {
  std::vector<float> scores;
  MF_TRY(tilt_axis_scores_finish(&s->ctx->c, &A->job, &scores));
  const int num = (int)A->cand.size(), nz = s->nz;
  if (scores_out) std::copy(scores.begin(), scores.end(), scores_out);
  int best = 0;
  float bs = 0.0f;
  for (int i = 0; i < num; ++i)
    if (bs < scores[i]) {
      bs = scores[i];
      best = i;
    }
  float axis = A->cand[best];
  if (axis < -45 && s->rot[0] == 0) axis += 180.0f;
  if (axis > 135) axis -= 180.0f;
  for (int i = 0; i < nz; ++i) s->rot[i] = axis;
  if (axis_out) *axis_out = axis;
  return MF_OK;
}

int tilt_axis(mf_series* s, float range, int num, float* axis_out, float* scores_out) {
  StageTimer timer(&s->ctx->c, kStageAxis);
  AxisSearch A;
  MF_TRY(axis_enqueue(s, range, num, 0, &A));
  MF_CHECK_CUDA(cudaStreamSynchronize(s->ctx->c.stream));
  return axis_finish(s, &A, axis_out, scores_out);
}

// ---------------------------------------------------------------------------
// FindOffset::DoIt (FindOffset.cu:85-238): offset_enqueue queues the moments of
// every (offset, tilt pair) (to the context's page-locked slot `slot`),
// offset_finish picks the offset once the stream has been synchronised.
int offset_enqueue(mf_series* s, int slot, OffsetJob* J) {
  Context* c = &s->ctx->c;
  cudaStream_t st = c->stream;
  const int nx = s->nx, ny = s->ny, nz = s->nz, bin = 4;
  const int xb = nx / bin / 2 * 2, yb = ny / bin / 2 * 2;
  if (xb < 2 || yb < 2) return set_error(MF_ERR_ARG, "find offset: image too small");
  const size_t bpix = (size_t)xb * yb;
  MF_TRY(s->upload_params());
  // device buffers are released stream-ordered on return, after the queued work
  DevBuf corr, d_pairs, d_out;
  MF_TRY(corr.alloc(sizeof(float) * bpix * nz));
  MF_TRY(launch_correct_bin(c, s->stack.as<float>(), s->stack_t.as<float>(),
                            nx, ny, nullptr, nz, s->d_sx.as<float>(),
                            s->d_sy.as<float>(), s->d_rot.as<float>(), 0, bin, 0,
                            corr.as<float>(), xb, bpix, st));
  const int num = kOffsetCount;
  std::vector<float> a = s->angles;
  std::vector<OffsetPair> pairs;
  std::vector<int>& first = J->first;
  first.assign(num + 1, 0);
  for (int n = 0; n < num; ++n) {
    float off = 0.0f + (n - num / 2) * 1.0f;
    for (int z = 0; z < nz; ++z) a[z] += off;
    int zt = frame_idx_from_tilt(nz, a.data(), 0.0f);
    first[n] = (int)pairs.size();
    for (int i = 0; i < nz; ++i) {
      if (i == zt) continue;
      int r = (i < zt) ? i + 1 : i - 1;
      double ds = std::cos(kD2R * a[r]) / std::cos(kD2R * a[i]);
      float m[3];
      stretch_matrix((float)ds, 0.0f, m);
      pairs.push_back(OffsetPair{r, i, m[0], m[1], m[2]});
    }
    for (int z = 0; z < nz; ++z) a[z] -= off;
  }
  first[num] = (int)pairs.size();
  const int np = (int)pairs.size();
  J->h_mom = (double*)c->pinned.get(slot, sizeof(double) * 6 * std::max(np, 1));
  if (!J->h_mom) return MF_ERR_NOMEM;
  MF_TRY(d_pairs.alloc(sizeof(OffsetPair) * np));
  MF_TRY(d_out.alloc(sizeof(double) * 6 * np));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_pairs.p, pairs.data(), sizeof(OffsetPair) * np,
                                cudaMemcpyHostToDevice, st));
  MF_TRY(offset_moments(c, corr.as<float>(), xb, yb, d_pairs.as<OffsetPair>(), np,
                        d_out.as<double>(), st));
  MF_CHECK_CUDA(cudaMemcpyAsync(J->h_mom, d_out.p, sizeof(double) * 6 * np,
                                cudaMemcpyDeviceToHost, st));
  return MF_OK;
}

int offset_finish(mf_series* s, OffsetJob* J, float* offset_out) {
  const int num = kOffsetCount;
  const std::vector<int>& first = J->first;
  const double* mom = J->h_mom;
  float maxcc = 0.0f, best = 0.0f;
  for (int n = 0; n < num; ++n) {
    float off = 0.0f + (n - num / 2) * 1.0f;
    float ccsum = 0.0f;
    int count = 0;
    for (int p = first[n]; p < first[n + 1]; ++p) {
      float f[6];
      for (int k = 0; k < 6; ++k) f[k] = (float)mom[(size_t)6 * p + k];
      for (int k = 0; k < 5; ++k) f[k] /= f[5];
      // the reference subtracts the mean itself, not its square (FindOffset.cu:222-223)
      double s1 = f[2] - f[0], s2 = f[3] - f[1];
      double cc = f[4] - f[0] * f[1];
      if (s1 < 0) s1 = 0;
      if (s2 < 0) s2 = 0;
      s1 = std::sqrt(s1);
      s2 = std::sqrt(s2);
      cc = cc / (s1 * s2 + 1e-30);
      if (cc < -1)
        cc = -1;
      else if (cc > 1)
        cc = 1;
      ccsum += (float)cc;
      count++;
    }
    float mcc = ccsum / count;
    if (mcc > maxcc) {
      maxcc = mcc;
      best = off;
    }
  }
  s->angle_offset += best;
  if (offset_out) *offset_out = best;
  return MF_OK;
}

int find_offset(mf_series* s, float* offset_out) {
  StageTimer timer(&s->ctx->c, kStageCoarse);
  OffsetJob J;
  MF_TRY(offset_enqueue(s, 0, &J));
  MF_CHECK_CUDA(cudaStreamSynchronize(s->ctx->c.stream));
  return offset_finish(s, &J, offset_out);
}

// ---------------------------------------------------------------------------
// ProjAlign::Setup / Setsize (ProjAlign.cpp:48-125) plus the precomputation
// that the reference repeats for every pass: processing order, neighbour
// ranges and the re-projection operators.
int projalign_setup(mf_series* s, float zshift, int align_z, int nproj) {
  StageTimer timer(&s->ctx->c, kStageSetup);
  Context* c = &s->ctx->c;
  cudaStream_t st = c->stream;
  if (nproj <= 0) return set_error(MF_ERR_ARG, "nproj must be > 0");
  ProjAlignState& P = s->pa;
  if (P.graph) {
    cudaGraphExecDestroy(P.graph);
    P.graph = nullptr;
  }
  P.ready = false;
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  int bx = (int)((float)nx / 2048.0f + 0.5f), by = (int)((float)ny / 2048.0f + 0.5f);
  P.bin = std::max(1, std::max(bx, by));
  P.xb = nx / P.bin / 2 * 2;
  P.yb = ny / P.bin / 2 * 2;
  P.pad = (P.xb / 2 + 1) * 2;
  P.cmp = P.pad / 2;
  P.thick = align_z / P.bin / 2 * 2;
  P.nproj = nproj;
  P.z0 = zshift;
  if (P.thick < 2) return set_error(MF_ERR_ARG, "slab thickness %d too small", P.thick);
  const int xb = P.xb, yb = P.yb;
  const size_t bpix = (size_t)xb * yb, ppix = (size_t)P.pad * yb;
  MF_TRY(P.corr.alloc(sizeof(float) * bpix * nz));
  MF_TRY(P.scratch.alloc(sizeof(float) * ppix * nz));
  MF_TRY(P.reproj.alloc(sizeof(float) * bpix));
  MF_TRY(P.ccbuf.alloc(sizeof(float) * ppix * 2));
  MF_TRY(P.part.alloc(sizeof(double2) * moment_parts(yb) * 2 + sizeof(float2) * kPeakParts));
  MF_TRY(P.stats.alloc(sizeof(float2) * 2));
  // the round-edge mask of MeaAlignProj (one geometry for every tilt and pass)
  MF_TRY(P.mask.alloc(sizeof(float) * bpix));
  MF_TRY(make_round_mask(c, xb, yb, (float)((P.pad / 2 - 1) * 2) * 0.5f, (float)yb * 0.5f,
                         (float)P.pad, (float)yb, 4.0f, P.mask.as<float>(), c->stream));
  // outward order (ProjAlign.cpp:151-176) and neighbour ranges
  P.zt = frame_idx_from_tilt(nz, s->angles.data(), 0.0f);
  std::vector<unsigned char> skip(nz, 1);
  skip[P.zt] = 0;
  P.order.clear();
  P.geom.clear();
  P.ops.ops.clear();
  for (int i = 1; i < nz; ++i) {
    for (int side = 0; side < 2; ++side) {
      int ip = side == 0 ? P.zt + i : P.zt - i;
      if (ip < 0 || ip >= nz) continue;
      int rg[2];
      find_proj_range(s->angles.data(), nz, skip.data(), ip, nproj, rg);
      if (rg[0] < 0 || rg[1] < 0)
        return set_error(MF_ERR_GEOMETRY,
                         "no already-aligned tilt within 20.5 degrees of tilt %d (%.2f)", ip,
                         s->angles[ip]);
      ReprojGeom g;
      reproj_geometry(s->angles.data(), ip, rg[0], rg[1], xb, yb, P.thick, &g);
      P.order.push_back(ip);
      P.geom.push_back(g);
      skip[ip] = 0;
    }
  }
  const int n = (int)P.order.size();
  MF_TRY(fill_bp_device(c, s->angles.data(), &P.geom, st));
  P.ytiles = (yb + kApplyTileY - 1) / kApplyTileY;
  MF_TRY(P.d_order.alloc(sizeof(int) * std::max(n, 1)));
  MF_TRY(P.d_err.alloc(sizeof(float) * nz));
  MF_TRY(P.d_z0.alloc(sizeof(float)));
  MF_TRY(P.d_maxerr.alloc(sizeof(float)));
  MF_TRY(P.d_meas.alloc(sizeof(float) * 2 * nz));
  P.bp_off.assign(n, 0);
  std::vector<float> bp;
  for (int k = 0; k < n; ++k) {
    P.bp_off[k] = bp.size();
    bp.insert(bp.end(), P.geom[k].bp.begin(), P.geom[k].bp.end());
  }
  MF_TRY(P.d_bp.alloc(sizeof(float) * std::max<size_t>(bp.size(), 1)));
  if (n > 0) {
    MF_CHECK_CUDA(cudaMemcpyAsync(P.d_order.p, P.order.data(), sizeof(int) * n,
                                  cudaMemcpyHostToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(P.d_bp.p, bp.data(), sizeof(float) * bp.size(),
                                  cudaMemcpyHostToDevice, st));
  }
  MF_CHECK_CUDA(cudaMemsetAsync(P.d_err.p, 0, sizeof(float) * nz, st));
  MF_CHECK_CUDA(cudaMemsetAsync(P.d_meas.p, 0, sizeof(float) * 2 * nz, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(P.d_z0.p, &P.z0, sizeof(float), cudaMemcpyHostToDevice, st));
  P.reproj_bytes = 0;
  P.reproj_fma = 0;
  P.prec = s->precision;
  if (P.prec != MF_PREC_FP32) {
    P.xpitch = (xb + 7) / 8 * 8;
    MF_TRY(P.corr16.alloc((size_t)2 * P.xpitch * yb * nz));
    MF_TRY(P.tflags.alloc(sizeof(int) * (size_t)nz * P.ytiles * kFlagParts));
    MF_TRY(P.d_tcerr.alloc(sizeof(int)));
    MF_CHECK_CUDA(cudaMemsetAsync(P.d_tcerr.p, 0, sizeof(int), st));
    P.tc_nb = tc_pick_rows(c, xb, yb);
    MF_TRY(tc_prepare(c, P.tc_nb));
    MF_TRY(tc_image_map(P.corr16.p, P.prec, xb, P.xpitch, yb, nz, P.tc_nb, &P.imgmap));
    MF_TRY(build_reproj_tc_ops(c, P.geom, P.prec, &P.tcops, st));
    P.reproj_bytes = P.tcops.bytes;
    P.reproj_fma = P.tcops.fma;
  } else if (P.method == 1) {
    MF_TRY(build_reproj_ops(c, P.geom, &P.ops, st));
    P.reproj_bytes = P.ops.bytes;
    P.reproj_fma = P.ops.fma;
    // the group apply with one job per held-out tilt; sentinel flags per tile of
    // the corrected stack send the tiles that need it to the exact path
    MF_TRY(P.tflags.alloc(sizeof(int) * (size_t)nz * P.ytiles * kFlagParts));
    std::vector<ApplyJob> jobs(std::max(n, 1));
    for (int k = 0; k < n; ++k) {
      const ReprojOpView& v = P.ops.ops[k];
      ApplyJob J{};
      J.tiles = v.tiles;
      J.colvalid = v.colvalid;
      J.corr = P.corr.as<float>();
      J.out = P.reproj.as<float>();
      J.xb = xb;
      J.yb = yb;
      J.ntiles = v.ntiles;
      jobs[k] = J;
    }
    MF_TRY(prepare_apply_group(c));
    MF_TRY(P.d_applyjobs.alloc(sizeof(ApplyJob) * jobs.size()));
    MF_CHECK_CUDA(cudaMemcpyAsync(P.d_applyjobs.p, jobs.data(), sizeof(ApplyJob) * jobs.size(),
                                  cudaMemcpyHostToDevice, st));
  } else {
    // compulsory traffic: the K neighbour images read once, the re-projection written
    for (int k = 0; k < n; ++k) P.reproj_bytes += 4.0 * (double)bpix * (P.geom[k].nk + 1);
  }
  // FFT plans
  MF_TRY(s->ctx->plan({0, xb, yb, (long long)nz * yb}, &P.rows_fwd_all));
  MF_TRY(s->ctx->plan({1, xb, yb, (long long)nz * yb}, &P.rows_inv_all));
  MF_TRY(s->ctx->plan({0, xb, yb, yb}, &P.rows_fwd_one));
  MF_TRY(s->ctx->plan({1, xb, yb, yb}, &P.rows_inv_one));
  MF_TRY(s->ctx->plan({2, xb, yb, 2}, &P.cc_fwd));
  MF_TRY(s->ctx->plan({3, xb, yb, 1}, &P.cc_inv));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  P.ready = true;
  return MF_OK;
}

// Queue one projection-matching pass (ProjAlign::DoItBin, ProjAlign.cpp:133-179).
static int pa_enqueue(mf_series* s) {
  Context* c = &s->ctx->c;
  cudaStream_t st = c->stream;
  ProjAlignState& P = s->pa;
  const int nz = s->nz, xb = P.xb, yb = P.yb, pad = P.pad, cmp = P.cmp;
  const size_t bpix = (size_t)xb * yb, ppix = (size_t)pad * yb;
  const int n = (int)P.order.size();
  float* corr = P.corr.as<float>();
  float* scratch = P.scratch.as<float>();
  float* cc = P.ccbuf.as<float>();
  double2* mpart = P.part.as<double2>();
  float2* ppart = reinterpret_cast<float2*>(mpart + moment_parts(yb) * 2);
  float2* stats = P.stats.as<float2>();
  // CorrTomoStack::DoIt: resample + bin + R-weight every tilt (CorrStack.cu:353-397)
  MF_TRY(launch_correct_bin(c, s->stack.as<float>(), s->stack_t.as<float>(),
                            s->nx, s->ny, nullptr, nz,
                            s->d_sx.as<float>(), s->d_sy.as<float>(), s->d_rot.as<float>(), 0,
                            P.bin, 1, scratch, pad, ppix, st));
  MF_CHECK_CUFFT(cufftExecR2C(P.rows_fwd_all, scratch, (cufftComplex*)scratch));
  MF_TRY(launch_rweight(c, (cufftComplex*)scratch, cmp, nz * yb, st));
  MF_CHECK_CUFFT(cufftExecC2R(P.rows_inv_all, (cufftComplex*)scratch, corr));
  const bool tc = P.prec != MF_PREC_FP32;
  const bool op32 = !tc && P.method == 1;
  if (tc)
    MF_TRY(launch_to_half(c, corr, xb, yb, nullptr, 0, nz, P.prec, P.corr16.p, P.xpitch,
                          P.tflags.as<int>(), st));
  else if (op32)
    MF_TRY(launch_flag_tiles(c, corr, xb, yb, nullptr, nz, P.tflags.as<int>(), st));
  // FitRotCenterZ + RemoveOffsetZ(-1)
  MF_TRY(fit_z0(c, nz, P.zt, s->d_angles.as<float>(), s->d_sx.as<float>(), s->d_sy.as<float>(),
                s->dev_sx64(), s->dev_sy64(), s->d_rot.as<float>(), P.d_z0.as<float>(), st));
  const bool prof = c->profiling && (int)P.events.size() >= 3 * n;
  for (int k = 0; k < n; ++k) {
    const int ip = P.order[k];
    const ReprojGeom& g = P.geom[k];
    float* reproj = P.reproj.as<float>();
    if (prof) MF_CHECK_CUDA(cudaEventRecord(P.events[3 * k], st));
    if (tc) {
      MF_TRY(launch_reproject_tc(c, P.tcops, P.tcops.ops[k], P.imgmap, P.tc_nb,
                                 P.d_tcerr.as<int>(), reproj, st));
      MF_TRY(launch_reproject_exact_flagged(c, corr, xb, yb, bpix, P.d_bp.as<float>() + P.bp_off[k],
                                            g.i0, g.nk, g.fcos, g.fsin, g.ray_len, g.thick,
                                            P.tflags.as<int>(), reproj, st));
    } else if (op32) {
      MF_TRY(launch_reproject_apply_group(c, P.ops, P.d_applyjobs.as<ApplyJob>() + k, nullptr, 1,
                                          P.ops.ops[k].ntiles, yb, st));
      MF_TRY(launch_reproject_exact_flagged(c, corr, xb, yb, bpix, P.d_bp.as<float>() + P.bp_off[k],
                                            g.i0, g.nk, g.fcos, g.fsin, g.ray_len, g.thick,
                                            P.tflags.as<int>(), reproj, st));
    } else {
      MF_TRY(launch_reproject_exact(c, corr, xb, yb, bpix, P.d_bp.as<float>() + P.bp_off[k], g.i0,
                                    g.nk, g.fcos, g.fsin, g.ray_len, g.thick, nullptr, reproj,
                                    st));
    }
    if (prof) MF_CHECK_CUDA(cudaEventRecord(P.events[3 * k + 1], st));
    // MeaAlignProj: PANorm both, FFT, filter, inverse FFT, peak
    const float mcx = (float)((pad / 2 - 1) * 2) * 0.5f, mcy = (float)yb * 0.5f;
    MF_TRY(norm_mask_pad(c, reproj, corr + (size_t)ip * bpix, xb, 0, xb, yb, pad, ppix, 2, 0, mcx,
                         mcy, (float)pad, (float)yb, 4.0f, P.mask.as<float>(), cc, mpart, stats,
                         st));
    MF_CHECK_CUFFT(cufftExecR2C(P.cc_fwd, cc, (cufftComplex*)cc));
    MF_TRY(xcorr_filter(c, (cufftComplex*)cc, 0, nullptr, (cufftComplex*)(cc + ppix), 0, 1, cmp,
                        yb, 500.0f, 1.0f, st));
    MF_CHECK_CUFFT(cufftExecC2R(P.cc_inv, (cufftComplex*)(cc + ppix), cc + ppix));
    MF_TRY(pa_peak_update(c, cc + ppix, pad, xb, yb, ppart, ip, s->nx, s->ny,
                          s->d_angles.as<float>(), s->d_sx.as<float>(), s->d_sy.as<float>(),
                          s->dev_sx64(), s->dev_sy64(), s->d_rot.as<float>(), P.d_z0.as<float>(),
                          P.d_err.as<float>(),
                          P.d_meas.as<float>(), st));
    // re-correct the aligned tilt (mCorrectProj)
    MF_TRY(launch_correct_bin(c, s->stack.as<float>(), s->stack_t.as<float>(),
                              s->nx, s->ny, P.d_order.as<int>() + k, 1,
                              s->d_sx.as<float>(), s->d_sy.as<float>(), s->d_rot.as<float>(), 0,
                              P.bin, 1, scratch, pad, ppix, st));
    MF_CHECK_CUFFT(cufftExecR2C(P.rows_fwd_one, scratch, (cufftComplex*)scratch));
    MF_TRY(launch_rweight(c, (cufftComplex*)scratch, cmp, yb, st));
    MF_CHECK_CUFFT(cufftExecC2R(P.rows_inv_one, (cufftComplex*)scratch, corr + (size_t)ip * bpix));
    if (tc)
      MF_TRY(launch_to_half(c, corr, xb, yb, P.d_order.as<int>() + k, 0, 1, P.prec, P.corr16.p,
                            P.xpitch, P.tflags.as<int>(), st));
    else if (op32)
      MF_TRY(launch_flag_tiles(c, corr, xb, yb, P.d_order.as<int>() + k, 1, P.tflags.as<int>(),
                               st));
    if (prof) MF_CHECK_CUDA(cudaEventRecord(P.events[3 * k + 2], st));
  }
  MF_TRY(max_err(c, P.d_err.as<float>(), P.d_order.as<int>(), n, P.d_maxerr.as<float>(), st));
  return MF_OK;
}

int projalign_doit(mf_series* s, float* max_err_out) {
  StageTimer timer(&s->ctx->c, kStagePass);
  ProjAlignState& P = s->pa;
  if (!P.ready) return set_error(MF_ERR_STATE, "projection matching is not set up");
  Context* c = &s->ctx->c;
  cudaStream_t st = c->stream;
  MF_TRY(s->upload_params());
  const int n = (int)P.order.size();
  if (c->profiling && (int)P.events.size() < 3 * n) {
    while ((int)P.events.size() < 3 * n) {
      cudaEvent_t e;
      MF_CHECK_CUDA(cudaEventCreate(&e));
      P.events.push_back(e);
    }
  }
  // Profiled passes run eagerly: events recorded by graph nodes cannot be timed.
  if (P.use_graph && !P.graph && !c->profiling) {
    // Capture once; the graph reads parameters from device memory, so every
    // later pass replays it unchanged.
    int64_t l0 = c->launches;
    cudaGraph_t g = nullptr;
    std::unique_lock<std::recursive_mutex> fft_lock(fft_mutex());
    MF_CHECK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = pa_enqueue(s);
    cudaError_t ec = cudaStreamEndCapture(st, &g);
    fft_lock.unlock();
    P.graph_kernels = c->launches - l0;
    c->launches = l0;
    if (rc != MF_OK || ec != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      P.use_graph = false;  // run eagerly from now on
    } else {
      cudaError_t ei = cudaGraphInstantiate(&P.graph, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) {
        cudaGetLastError();
        P.graph = nullptr;
        P.use_graph = false;
      }
    }
  }
  if (P.graph && !c->profiling) {
    MF_CHECK_CUDA(cudaGraphLaunch(P.graph, st));
    c->launches += P.graph_kernels;
  } else {
    MF_TRY(pa_enqueue(s));
  }
  float res[2];
  int tcerr = 0;
  MF_CHECK_CUDA(cudaMemcpyAsync(&res[0], P.d_maxerr.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(&res[1], P.d_z0.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  if (P.prec != MF_PREC_FP32)
    MF_CHECK_CUDA(cudaMemcpyAsync(&tcerr, P.d_tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  MF_TRY(s->download_shifts());
  if (tcerr != 0)
    return set_error(MF_ERR_CUDA, "tensor-core re-projection pipeline stalled (code %d)", tcerr);
  P.z0 = res[1];
  if (c->profiling && (int)P.events.size() >= 3 * n) {
    for (int k = 0; k < n; ++k) {
      float a = 0.0f, b = 0.0f;
      MF_CHECK_CUDA(cudaEventElapsedTime(&a, P.events[3 * k], P.events[3 * k + 1]));
      MF_CHECK_CUDA(cudaEventElapsedTime(&b, P.events[3 * k + 1], P.events[3 * k + 2]));
      c->stage[0] += a;
      c->stage[2] += b;
    }
    c->stage[1] += n;
    c->stage[3] += 1;
    c->stage[4] += P.reproj_bytes;
    c->stage[5] += P.reproj_fma;
  }
  if (max_err_out) *max_err_out = res[0];
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Process::mCoarseAlign (Process.cpp:238-270)
int coarse_align(mf_series* s, float pitch_angle, float offset) {
  if (pitch_angle == 0) {
    s->tr.ready = false;
    for (int i = 1; i <= 3; ++i) {
      float e, ax;
      MF_TRY(transform_doit(s, &e));
      MF_TRY(tilt_axis(s, 180.0f / i, 100, &ax, nullptr));
    }
  } else {
    for (int i = 0; i < s->nz; ++i) s->rot[i] = pitch_angle;
  }
  if (offset == 0) {
    float o;
    MF_TRY(find_offset(s, &o));
  } else {
    s->angle_offset = offset;
  }
  for (int z = 0; z < s->nz; ++z) s->angles[z] += s->angle_offset;
  return MF_OK;
}

// The same for n series of one context, stage by stage: every stage is queued for
// all series (results to page-locked slots 0..n-1) before one wait, so the GPU
// runs the series' work back to back instead of idling at a host round trip per
// series.  Each series' arithmetic and decisions are those of coarse_align.
int transform_many(mf_series* const* ser, int n) {
  StageTimer timer(&ser[0]->ctx->c, kStageCoarse);
  std::vector<TransformJob> J(n);
  for (int i = 0; i < n; ++i) MF_TRY(transform_enqueue(ser[i], i, &J[i]));
  MF_CHECK_CUDA(cudaStreamSynchronize(ser[0]->ctx->c.stream));
  for (int i = 0; i < n; ++i) MF_TRY(transform_finish(ser[i], &J[i], nullptr));
  return MF_OK;
}

int tilt_axis_many(mf_series* const* ser, int n, float range, int num) {
  StageTimer timer(&ser[0]->ctx->c, kStageAxis);
  std::vector<AxisSearch> A(n);
  for (int i = 0; i < n; ++i) MF_TRY(axis_enqueue(ser[i], range, num, i, &A[i]));
  MF_CHECK_CUDA(cudaStreamSynchronize(ser[0]->ctx->c.stream));
  for (int i = 0; i < n; ++i) MF_TRY(axis_finish(ser[i], &A[i], nullptr, nullptr));
  return MF_OK;
}

int coarse_align_many(mf_series* const* ser, int n, float pitch_angle, float offset) {
  if (n < 1) return MF_OK;
  for (int i = 1; i < n; ++i)
    if (ser[i]->ctx != ser[0]->ctx) return set_error(MF_ERR_ARG, "series of different contexts");
  if (pitch_angle == 0) {
    for (int i = 0; i < n; ++i) ser[i]->tr.ready = false;
    for (int k = 1; k <= 3; ++k) {
      MF_TRY(transform_many(ser, n));
      MF_TRY(tilt_axis_many(ser, n, 180.0f / k, 100));
    }
  } else {
    for (int i = 0; i < n; ++i)
      for (int z = 0; z < ser[i]->nz; ++z) ser[i]->rot[z] = pitch_angle;
  }
  if (offset == 0) {
    StageTimer timer(&ser[0]->ctx->c, kStageCoarse);
    std::vector<OffsetJob> J(n);
    for (int i = 0; i < n; ++i) MF_TRY(offset_enqueue(ser[i], i, &J[i]));
    MF_CHECK_CUDA(cudaStreamSynchronize(ser[0]->ctx->c.stream));
    for (int i = 0; i < n; ++i) MF_TRY(offset_finish(ser[i], &J[i], nullptr));
  } else {
    for (int i = 0; i < n; ++i) ser[i]->angle_offset = offset;
  }
  for (int i = 0; i < n; ++i)
    for (int z = 0; z < ser[i]->nz; ++z) ser[i]->angles[z] += ser[i]->angle_offset;
  return MF_OK;
}

// Process::mProjAlign + ProjAlignOnce (Process.cpp:272-319)
int proj_align(mf_series* s, float zshift, int align_z, int nproj, int* passes) {
  for (int i = 0; i < s->nz; ++i) {
    s->sx[i] = 0.0f;
    s->sy[i] = 0.0f;
  }
  MF_TRY(projalign_setup(s, zshift, align_z, nproj));
  int np = 0;
  auto once = [&]() -> int {
    float last;
    MF_TRY(projalign_doit(s, &last));
    np++;
    for (int i = 1; i < 10; ++i) {
      float e;
      MF_TRY(projalign_doit(s, &e));
      np++;
      if (e <= last) {
        if (e < 2.0f) break;
        last = e;
      }
    }
    return MF_OK;
  };
  MF_TRY(once());
  for (int i = 1; i <= 4; ++i) {
    float ax;
    MF_TRY(tilt_axis(s, 20.0f / i, 100, &ax, nullptr));
    if (i == 1) MF_TRY(once());
  }
  MF_TRY(once());
  if (passes) *passes = np;
  return MF_OK;
}

// Process::CorrectStack (Process.cpp:329-372) into device memory.
int correct_stack_device(mf_series* s, int out_bin, float* d_out) {
  StageTimer timer(&s->ctx->c, kStageFinal);
  Context* c = &s->ctx->c;
  if (out_bin < 1) return set_error(MF_ERR_ARG, "output binning must be >= 1");
  int xo = s->nx / out_bin / 2 * 2, yo = s->ny / out_bin / 2 * 2;
  if (xo < 2 || yo < 2) return set_error(MF_ERR_ARG, "output binning too large");
  MF_TRY(s->upload_params());
  MF_TRY(launch_correct_bin(c, s->stack.as<float>(), s->stack_t.as<float>(),
                            s->nx, s->ny, nullptr, s->nz,
                            s->d_sx.as<float>(), s->d_sy.as<float>(), s->d_rot.as<float>(), 0,
                            out_bin, 1, d_out, xo, (size_t)xo * yo, c->stream));
  return MF_OK;
}

}  // namespace mf
