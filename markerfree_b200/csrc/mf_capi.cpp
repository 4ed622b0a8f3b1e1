// extern "C" entry points (include/markerfree.h).
#include <algorithm>
#include <cstring>
#include <new>

#include "mf_series.hpp"
#include "mf_xcorr.hpp"

namespace mf {
const char* last_error();
}

using namespace mf;

#define MF_GUARD_BEGIN try {
#define MF_GUARD_END                                                      \
  }                                                                       \
  catch (const std::bad_alloc&) {                                         \
    return set_error(MF_ERR_NOMEM, "host allocation failed");             \
  }                                                                       \
  catch (...) {                                                           \
    return set_error(MF_ERR_STATE, "unexpected exception in the library"); \
  }

static int use_device(mf_context* ctx) {
  if (!ctx) return set_error(MF_ERR_ARG, "null context");
  MF_CHECK_CUDA(cudaSetDevice(ctx->c.gpu));
  set_alloc_stream(ctx->c.stream);
  return MF_OK;
}

static mf_context::Scratch* scratch_of(mf_context* ctx) { return &ctx->scratch; }

extern "C" {

MF_API const char* mf_last_error(void) { return mf::last_error(); }
MF_API const char* mf_version(void) { return "markerfree-b200 0.1 (sm_100a)"; }

MF_API void mf_debug_fail_device_allocations(int64_t first, int64_t count) {
  fail_device_allocations(first, count);
}

MF_API int mf_context_create(int gpu, mf_context** out) {
  MF_GUARD_BEGIN
  if (!out) return set_error(MF_ERR_ARG, "null output pointer");
  *out = nullptr;
  int n = 0;
  MF_CHECK_CUDA(cudaGetDeviceCount(&n));
  if (gpu < 0 || gpu >= n) return set_error(MF_ERR_ARG, "GPU %d not present (%d visible)", gpu, n);
  MF_CHECK_CUDA(cudaSetDevice(gpu));
  mf_context* ctx = new mf_context();
  ctx->c.gpu = gpu;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, gpu) == cudaSuccess) ctx->c.sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return set_error(MF_ERR_CUDA, "cudaStreamCreate failed");
  }
  // keep freed device memory in the pool for the next series
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, gpu) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  *out = ctx;
  return MF_OK;
  MF_GUARD_END
}

MF_API void mf_context_destroy(mf_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->c.gpu);
  cudaStreamSynchronize(ctx->c.stream);
  set_sync_free(true);
  delete ctx;
  set_sync_free(false);
  set_alloc_stream(nullptr);
}

MF_API int mf_context_sync(mf_context* ctx) {
  MF_TRY(use_device(ctx));
  MF_CHECK_CUDA(cudaStreamSynchronize(ctx->c.stream));
  return MF_OK;
}

MF_API int64_t mf_context_kernel_launches(mf_context* ctx) { return ctx ? ctx->c.launches : 0; }

MF_API int mf_context_set_profiling(mf_context* ctx, int on) {
  if (!ctx) return set_error(MF_ERR_ARG, "null context");
  ctx->c.profiling = on != 0;
  return MF_OK;
}

MF_API int mf_context_stage_times(mf_context* ctx, double* out6) {
  if (!ctx || !out6) return set_error(MF_ERR_ARG, "null argument");
  for (int i = 0; i < 6; ++i) {
    out6[i] = ctx->c.stage[i];
    ctx->c.stage[i] = 0.0;
  }
  return MF_OK;
}

MF_API int mf_context_stage_breakdown(mf_context* ctx, double* out10) {
  if (!ctx || !out10) return set_error(MF_ERR_ARG, "null argument");
  static_assert(kStages == 10, "mf_context_stage_breakdown returns 10 values");
  for (int i = 0; i < kStages; ++i) {
    out10[i] = ctx->c.breakdown[i];
    ctx->c.breakdown[i] = 0.0;
  }
  return MF_OK;
}

MF_API int mf_device_cos_sin(mf_context* ctx, const float* x, int n, float* c, float* s) {
  MF_GUARD_BEGIN
  if (!ctx || n < 0 || (n > 0 && (!x || !c || !s))) return set_error(MF_ERR_ARG, "bad argument");
  if (n == 0) return MF_OK;
  MF_TRY(use_device(ctx));
  cudaStream_t st = ctx->c.stream;
  DevBuf d;
  MF_TRY(d.alloc(sizeof(float) * 3 * (size_t)n));
  float* dx = d.as<float>();
  MF_CHECK_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  MF_TRY(device_cos_sin(&ctx->c, dx, n, dx + n, dx + 2 * (size_t)n, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(c, dx + n, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(s, dx + 2 * (size_t)n, sizeof(float) * n, cudaMemcpyDeviceToHost,
                                st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
  MF_GUARD_END
}

MF_API void* mf_context_stream(mf_context* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

MF_API int mf_context_set_tc_rows(mf_context* ctx, int rows) {
  if (!ctx) return set_error(MF_ERR_ARG, "null context");
  if (rows != 0 && rows != 64 && rows != 128 && rows != 256)
    return set_error(MF_ERR_ARG, "tensor-core tile rows must be 0, 64, 128 or 256 (got %d)", rows);
  ctx->c.tc_rows = rows;
  return MF_OK;
}

MF_API int mf_context_tc_tuning(mf_context* ctx, double* out, int max_rows, int* n) {
  if (!ctx || !n || max_rows < 0 || (max_rows > 0 && !out))
    return set_error(MF_ERR_ARG, "bad argument");
  const auto& t = ctx->c.tc_tuned;
  const auto& ms = ctx->c.tc_tuned_ms;
  *n = (int)t.size();
  for (int i = 0; i < (int)t.size() && i < max_rows; ++i) {
    for (int k = 0; k < 5; ++k) out[8 * i + k] = t[i][k];
    for (int k = 0; k < 3; ++k) out[8 * i + 5 + k] = i < (int)ms.size() ? ms[i][k] : 0.0;
  }
  return MF_OK;
}

// ---------------------------------------------------------------------------
static int series_create_common(mf_context* ctx, const float* raw, bool raw_on_device, int nx,
                                int ny, int nz, const float* file_angles, mf_series** out,
                                bool preprocess = true) {
  if (!out) return set_error(MF_ERR_ARG, "null output pointer");
  *out = nullptr;
  MF_TRY(use_device(ctx));
  if (!raw || !file_angles) return set_error(MF_ERR_ARG, "null stack or angles");
  if (nx < 8 || ny < 8 || nz < 2)
    return set_error(MF_ERR_ARG, "stack %d x %d x %d too small (need >= 8 x 8 x 2)", nx, ny, nz);
  StageTimer timer(&ctx->c, kStagePrep);
  mf_series* s = new mf_series();
  int rc = series_init(s, ctx, nx, ny, nz, file_angles);
  size_t pix = (size_t)nx * ny;
  if (rc == MF_OK) rc = s->stack.alloc(sizeof(float) * pix * nz);
  if (rc == MF_OK) {
    // SetPositive writes slice a to index nz-1-a when the angles descend
    bool rev = preprocess && file_angles[0] > file_angles[1];
    cudaStream_t st = ctx->c.stream;
    for (int a = 0; a < nz && rc == MF_OK; ++a) {
      int i = rev ? nz - 1 - a : a;
      cudaError_t e = cudaMemcpyAsync(s->stack.as<float>() + (size_t)i * pix, raw + (size_t)a * pix,
                                      sizeof(float) * pix,
                                      raw_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                      st);
      if (e != cudaSuccess) rc = set_error(MF_ERR_CUDA, "stack upload: %s", cudaGetErrorString(e));
    }
  }
  if (rc == MF_OK && preprocess)
    rc = preprocess_device(&ctx->c, s->stack.as<float>(), nx, ny, nz, file_angles, ctx->c.stream);
  // the column-major copy read by the resampling and the tilt-axis search
  if (rc == MF_OK) rc = s->stack_t.alloc(sizeof(float) * pix * nz);
  if (rc == MF_OK) rc = s->d_neg.alloc(sizeof(int) * nz);
  if (rc == MF_OK)
    rc = transpose_stack(&ctx->c, s->stack.as<float>(), nx, ny, nz, s->stack_t.as<float>(),
                         s->d_neg.as<int>(), ctx->c.stream);
  if (rc != MF_OK) {
    delete s;
    return rc;
  }
  *out = s;
  return MF_OK;
}

MF_API int mf_series_create(mf_context* ctx, const float* raw, int nx, int ny, int nz,
                            const float* file_angles, mf_series** out) {
  MF_GUARD_BEGIN
  return series_create_common(ctx, raw, false, nx, ny, nz, file_angles, out);
  MF_GUARD_END
}

MF_API int mf_series_create_device(mf_context* ctx, const float* d_raw, int nx, int ny, int nz,
                                   const float* file_angles, mf_series** out) {
  MF_GUARD_BEGIN
  return series_create_common(ctx, d_raw, true, nx, ny, nz, file_angles, out);
  MF_GUARD_END
}

MF_API int mf_series_create_preprocessed(mf_context* ctx, const float* stack, int nx, int ny,
                                         int nz, const float* angles, mf_series** out) {
  MF_GUARD_BEGIN
  if (angles)
    for (int z = 1; z < nz; ++z)
      if (!(angles[z] > angles[z - 1]))
        return set_error(MF_ERR_ARG, "a pre-processed stack is in ascending angle order "
                                     "(angle %d is %.2f after %.2f)", z, angles[z], angles[z - 1]);
  return series_create_common(ctx, stack, false, nx, ny, nz, angles, out, false);
  MF_GUARD_END
}

MF_API void mf_series_destroy(mf_series* s) {
  if (!s) return;
  // buffers go back to the pool in the order of the stream of the series' current
  // context (a served series may have been prepared on another worker's stream)
  cudaSetDevice(s->gpu);
  set_free_stream(s->ctx ? s->ctx->c.stream : nullptr);
  delete s;
  set_free_stream(nullptr);
}

MF_API int mf_series_set_precision(mf_series* s, mf_precision p) {
  if (!s) return set_error(MF_ERR_ARG, "null series");
  if (p != MF_PREC_FP32 && p != MF_PREC_BF16 && p != MF_PREC_FP16)
    return set_error(MF_ERR_ARG, "unknown precision %d", (int)p);
  if (s->precision != p && s->pa.ready) {
    // the operators and buffers of the set-up pass belong to the old precision
    if (s->pa.graph) cudaGraphExecDestroy(s->pa.graph);
    s->pa.graph = nullptr;
    s->pa.ready = false;
  }
  s->precision = p;
  return MF_OK;
}

MF_API int mf_series_get_stack(mf_series* s, float* out) {
  if (!s || !out) return set_error(MF_ERR_ARG, "null argument");
  MF_TRY(use_device(s->ctx));
  MF_CHECK_CUDA(cudaMemcpyAsync(out, s->stack.p, sizeof(float) * (size_t)s->nx * s->ny * s->nz,
                                cudaMemcpyDeviceToHost, s->ctx->c.stream));
  MF_CHECK_CUDA(cudaStreamSynchronize(s->ctx->c.stream));
  return MF_OK;
}

MF_API int mf_series_set_angles(mf_series* s, const float* a) {
  if (!s || !a) return set_error(MF_ERR_ARG, "null argument");
  s->angles.assign(a, a + s->nz);
  return MF_OK;
}

MF_API int mf_series_get_angles(mf_series* s, float* a) {
  if (!s || !a) return set_error(MF_ERR_ARG, "null argument");
  memcpy(a, s->angles.data(), sizeof(float) * s->nz);
  return MF_OK;
}

MF_API int mf_series_set_param(mf_series* s, const mf_align_param* p) {
  if (!s || !p || !p->shift_x || !p->shift_y || !p->rotate)
    return set_error(MF_ERR_ARG, "null argument");
  s->sx.assign(p->shift_x, p->shift_x + s->nz);
  s->sy.assign(p->shift_y, p->shift_y + s->nz);
  s->rot.assign(p->rotate, p->rotate + s->nz);
  s->angle_offset = p->angle_offset;
  return MF_OK;
}

MF_API int mf_series_get_param(mf_series* s, mf_align_param* p) {
  if (!s || !p || !p->shift_x || !p->shift_y || !p->rotate)
    return set_error(MF_ERR_ARG, "null argument");
  memcpy(p->shift_x, s->sx.data(), sizeof(float) * s->nz);
  memcpy(p->shift_y, s->sy.data(), sizeof(float) * s->nz);
  memcpy(p->rotate, s->rot.data(), sizeof(float) * s->nz);
  p->angle_offset = s->angle_offset;
  return MF_OK;
}

// ---------------------------------------------------------------------------
MF_API int mf_transform_doit(mf_series* s, float* max_err) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return transform_doit(s, max_err);
  MF_GUARD_END
}

MF_API int mf_tilt_axis(mf_series* s, float range, int num, float* axis_out) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return tilt_axis(s, range, num, axis_out, nullptr);
  MF_GUARD_END
}

MF_API int mf_tilt_axis_scores(mf_series* s, float range, int num, float* axis_out,
                               float* scores) {
  MF_GUARD_BEGIN
  if (!s || !scores) return set_error(MF_ERR_ARG, "null argument");
  MF_TRY(use_device(s->ctx));
  return tilt_axis(s, range, num, axis_out, scores);
  MF_GUARD_END
}

MF_API int mf_find_offset(mf_series* s, float* offset_out) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return find_offset(s, offset_out);
  MF_GUARD_END
}

MF_API int mf_projalign_setup(mf_series* s, float zshift, int align_z, int nproj) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return projalign_setup(s, zshift, align_z, nproj);
  MF_GUARD_END
}

MF_API int mf_projalign_doit(mf_series* s, float* max_err) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return projalign_doit(s, max_err);
  MF_GUARD_END
}

MF_API int mf_projalign_z0(mf_series* s, float* z0) {
  if (!s || !z0) return set_error(MF_ERR_ARG, "null argument");
  if (!s->pa.ready) return set_error(MF_ERR_STATE, "projection matching is not set up");
  *z0 = s->pa.z0;
  return MF_OK;
}

MF_API int mf_projalign_measured(mf_series* s, float* xy) {
  MF_GUARD_BEGIN
  if (!s || !xy) return set_error(MF_ERR_ARG, "null argument");
  if (!s->pa.ready) return set_error(MF_ERR_STATE, "projection matching is not set up");
  MF_TRY(use_device(s->ctx));
  cudaStream_t st = s->ctx->c.stream;
  MF_CHECK_CUDA(cudaMemcpyAsync(xy, s->pa.d_meas.p, sizeof(float) * 2 * s->nz,
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
  MF_GUARD_END
}

MF_API int mf_coarse_align(mf_series* s, float pitch_angle, float offset) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return coarse_align(s, pitch_angle, offset);
  MF_GUARD_END
}

MF_API int mf_proj_align(mf_series* s, float zshift, int align_z, int nproj, int* passes) {
  MF_GUARD_BEGIN
  if (!s) return set_error(MF_ERR_ARG, "null series");
  MF_TRY(use_device(s->ctx));
  return proj_align(s, zshift, align_z, nproj, passes);
  MF_GUARD_END
}

MF_API void mf_binned_size(int nx, int ny, int bin, int* xb, int* yb) {
  if (bin < 1) bin = 1;
  if (xb) *xb = nx / bin / 2 * 2;
  if (yb) *yb = ny / bin / 2 * 2;
}

MF_API int mf_correct_stack(mf_series* s, int out_bin, float* host_out) {
  MF_GUARD_BEGIN
  if (!s || !host_out) return set_error(MF_ERR_ARG, "null argument");
  MF_TRY(use_device(s->ctx));
  int xo, yo;
  mf_binned_size(s->nx, s->ny, out_bin, &xo, &yo);
  size_t n = (size_t)xo * yo * s->nz;
  DevBuf out;
  MF_TRY(out.alloc(sizeof(float) * n));
  MF_TRY(correct_stack_device(s, out_bin, out.as<float>()));
  MF_CHECK_CUDA(cudaMemcpyAsync(host_out, out.p, sizeof(float) * n, cudaMemcpyDeviceToHost,
                                s->ctx->c.stream));
  MF_CHECK_CUDA(cudaStreamSynchronize(s->ctx->c.stream));
  return MF_OK;
  MF_GUARD_END
}

static int align_common(mf_context* ctx, const float* raw, bool on_device, int nx, int ny, int nz,
                        const float* file_angles, const mf_options* opt, mf_align_param* param,
                        float* out, int* passes) {
  if (!opt || !param) return set_error(MF_ERR_ARG, "null options or parameters");
  if (opt->nproj <= 0) return set_error(MF_ERR_ARG, "nProj must be > 0.");
  if (opt->out_bin < 1) return set_error(MF_ERR_ARG, "output binning must be >= 1");
  if (opt->precision != MF_PREC_FP32 && opt->precision != MF_PREC_BF16 &&
      opt->precision != MF_PREC_FP16)
    return set_error(MF_ERR_ARG, "unknown precision %d", opt->precision);
  mf_series* s = nullptr;
  MF_TRY(series_create_common(ctx, raw, on_device, nx, ny, nz, file_angles, &s));
  s->precision = (mf_precision)opt->precision;
  int rc = MF_OK;
  int np = 0;
  if (opt->align_z != 0) {
    rc = coarse_align(s, opt->pitch_angle, opt->offset);
    if (rc == MF_OK) rc = proj_align(s, opt->zshift, opt->align_z, opt->nproj, &np);
  }
  if (rc == MF_OK && out) {
    if (on_device) {
      rc = correct_stack_device(s, opt->out_bin, out);
      if (rc == MF_OK && cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
        rc = set_error(MF_ERR_CUDA, "stream synchronize failed");
    } else {
      rc = mf_correct_stack(s, opt->out_bin, out);
    }
  }
  if (rc == MF_OK) rc = mf_series_get_param(s, param);
  if (passes) *passes = np;
  mf_series_destroy(s);
  return rc;
}

MF_API int mf_align(mf_context* ctx, const float* raw, int nx, int ny, int nz,
                    const float* file_angles, const mf_options* opt, mf_align_param* param,
                    float* aligned_out, int* passes) {
  MF_GUARD_BEGIN
  return align_common(ctx, raw, false, nx, ny, nz, file_angles, opt, param, aligned_out, passes);
  MF_GUARD_END
}

MF_API int mf_align_device(mf_context* ctx, const float* d_raw, int nx, int ny, int nz,
                           const float* file_angles, const mf_options* opt, mf_align_param* param,
                           float* d_aligned_out, int* passes) {
  MF_GUARD_BEGIN
  return align_common(ctx, d_raw, true, nx, ny, nz, file_angles, opt, param, d_aligned_out,
                      passes);
  MF_GUARD_END
}

}  // extern "C"

namespace {

// File samples of MRC mode 0 (8-bit), 1 (16-bit) or 2 (float) to float, as
// mrcstack.cpp:56-116 converts them on the host.
__global__ void k_mrc_to_float(const void* __restrict__ src, int mode, size_t n,
                               float* __restrict__ dst) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float v;
    if (mode == 0)
      v = (float)static_cast<const unsigned char*>(src)[i];
    else if (mode == 1)
      v = (float)static_cast<const short*>(src)[i];
    else
      v = static_cast<const float*>(src)[i];
    dst[i] = v;
  }
}

// Two page-locked host buffers for streaming between a file and the device.
struct PinnedPair {
  void* p[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int init(size_t bytes) {
    for (int k = 0; k < 2; ++k) {
      MF_CHECK_CUDA(cudaHostAlloc(&p[k], bytes, cudaHostAllocDefault));
      MF_CHECK_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    }
    return MF_OK;
  }
  ~PinnedPair() {
    for (int k = 0; k < 2; ++k) {
      if (ev[k]) cudaEventSynchronize(ev[k]);
      if (ev[k]) cudaEventDestroy(ev[k]);
      if (p[k]) cudaFreeHost(p[k]);
    }
    cudaGetLastError();
  }
};

struct FileCloser {
  FILE* f = nullptr;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

constexpr size_t kStreamChunk = (size_t)64 << 20;  // bytes per streamed block of slices

// Read the stack of an MRC file into d_raw (float, file order): whole slices in
// blocks of about kStreamChunk bytes, each read into one of two pinned buffers
// while the other one's block is copied to the device (and converted there for
// modes 0 and 1).
int upload_mrc(mf_context* ctx, FILE* f, int nx, int ny, int nz, int mode, float* d_raw) {
  cudaStream_t st = ctx->c.stream;
  const size_t pix = (size_t)nx * ny, psize = mode == 0 ? 1 : (mode == 1 ? 2 : 4);
  const size_t slice = pix * psize;
  const int per = (int)std::max<size_t>(1, kStreamChunk / slice);
  PinnedPair pin;
  MF_TRY(pin.init(slice * per));
  DevBuf stage[2];
  if (mode != 2)
    for (int k = 0; k < 2; ++k) MF_TRY(stage[k].alloc(slice * per));
  for (int z0 = 0, c = 0; z0 < nz; z0 += per, ++c) {
    const int k = c & 1, n = std::min(per, nz - z0);
    MF_CHECK_CUDA(cudaEventSynchronize(pin.ev[k]));  // the block that used this buffer is done
    if (fread(pin.p[k], 1, slice * n, f) != slice * n)
      return set_error(MF_ERR_FORMAT, "MRC file is truncated at slice %d", z0);
    float* dst = d_raw + (size_t)z0 * pix;
    if (mode == 2) {
      MF_CHECK_CUDA(cudaMemcpyAsync(dst, pin.p[k], slice * n, cudaMemcpyHostToDevice, st));
    } else {
      MF_CHECK_CUDA(cudaMemcpyAsync(stage[k].p, pin.p[k], slice * n, cudaMemcpyHostToDevice, st));
      k_mrc_to_float<<<ctx->c.sm_count * 4, 256, 0, st>>>(stage[k].p, mode, pix * n, dst);
      ctx->c.launches++;
      MF_CHECK_CUDA(cudaGetLastError());
    }
    MF_CHECK_CUDA(cudaEventRecord(pin.ev[k], st));
  }
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// Write the aligned stack d_out (nz x yo x xo float) as an MRC file: the header
// from the middle slice, then blocks of slices, each copied from the device into
// one pinned buffer while the previous block is written from the other.
int download_mrc(mf_context* ctx, const float* d_out, int xo, int yo, int nz, const char* path) {
  cudaStream_t st = ctx->c.stream;
  const size_t pix = (size_t)xo * yo, slice = pix * sizeof(float);
  const int per = (int)std::max<size_t>(1, kStreamChunk / slice);
  PinnedPair pin;
  MF_TRY(pin.init(slice * per));
  // header: statistics of the middle slice (mf_mrc_write's rule)
  const int zm = (int)(nz * .5);
  MF_CHECK_CUDA(cudaMemcpyAsync(pin.p[0], d_out + (size_t)zm * pix, slice, cudaMemcpyDeviceToHost,
                                st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  unsigned char hdr[1024];
  mrc_float_header(static_cast<const float*>(pin.p[0]), xo, yo, nz, hdr);
  FileCloser fc;
  fc.f = fopen(path, "wb");
  if (!fc.f) return set_error(MF_ERR_IO, "cannot open %s for writing", path);
  if (fwrite(hdr, 1, sizeof(hdr), fc.f) != sizeof(hdr))
    return set_error(MF_ERR_IO, "write failed on %s", path);
  const int nblk = (nz + per - 1) / per;
  auto issue = [&](int c) -> int {
    const int z0 = c * per, n = std::min(per, nz - z0);
    MF_CHECK_CUDA(cudaMemcpyAsync(pin.p[c & 1], d_out + (size_t)z0 * pix, slice * n,
                                  cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaEventRecord(pin.ev[c & 1], st));
    return MF_OK;
  };
  MF_TRY(issue(0));
  for (int c = 0; c < nblk; ++c) {
    if (c + 1 < nblk) MF_TRY(issue(c + 1));  // its buffer's previous block was written
    MF_CHECK_CUDA(cudaEventSynchronize(pin.ev[c & 1]));
    const size_t n = (size_t)std::min(per, nz - c * per);
    if (fwrite(pin.p[c & 1], 1, slice * n, fc.f) != slice * n)
      return set_error(MF_ERR_IO, "write failed on %s", path);
  }
  const int rc = fclose(fc.f);
  fc.f = nullptr;
  if (rc != 0) return set_error(MF_ERR_IO, "write failed on %s", path);
  return MF_OK;
}

}  // namespace

extern "C" {

MF_API int mf_align_file(mf_context* ctx, const char* in_mrc, const float* file_angles,
                         const mf_options* opt, mf_align_param* param, const char* out_mrc,
                         int* passes) {
  MF_GUARD_BEGIN
  if (!in_mrc || !file_angles || !opt || !param) return set_error(MF_ERR_ARG, "null argument");
  MF_TRY(use_device(ctx));
  FileCloser in;
  int nx = 0, ny = 0, nz = 0, mode = 0;
  MF_TRY(mrc_open_stack(in_mrc, &in.f, &nx, &ny, &nz, &mode));
  DevBuf raw;
  MF_TRY(raw.alloc(sizeof(float) * (size_t)nx * ny * nz));
  MF_TRY(upload_mrc(ctx, in.f, nx, ny, nz, mode, raw.as<float>()));
  fclose(in.f);
  in.f = nullptr;
  int xo = 0, yo = 0;
  mf_binned_size(nx, ny, std::max(1, opt->out_bin), &xo, &yo);
  DevBuf out;
  if (out_mrc) MF_TRY(out.alloc(sizeof(float) * (size_t)xo * yo * nz));
  MF_TRY(align_common(ctx, raw.as<float>(), true, nx, ny, nz, file_angles, opt, param,
                      out_mrc ? out.as<float>() : nullptr, passes));
  raw.release();
  if (out_mrc) MF_TRY(download_mrc(ctx, out.as<float>(), xo, yo, nz, out_mrc));
  return MF_OK;
  MF_GUARD_END
}

// ---------------------------------------------------------------------------
MF_API int mf_dev_correct_proj(mf_context* ctx, const float* d_proj, int nx, int ny,
                               float shift_x, float shift_y, float tilt_axis, int only_shift,
                               int bin, int random_fill, int rweight, float* d_out) {
  MF_GUARD_BEGIN
  MF_TRY(use_device(ctx));
  if (!d_proj || !d_out || bin < 1) return set_error(MF_ERR_ARG, "invalid argument");
  int xb = nx / bin / 2 * 2, yb = ny / bin / 2 * 2;
  if (xb < 2 || yb < 2) return set_error(MF_ERR_ARG, "image too small for binning %d", bin);
  cudaStream_t st = ctx->c.stream;
  if (!rweight)
    return launch_correct_one(&ctx->c, d_proj, nx, ny, shift_x, shift_y, tilt_axis, only_shift,
                              bin, random_fill, d_out, xb, st);
  int pad = (xb / 2 + 1) * 2, cmp = xb / 2 + 1;
  mf_context::Scratch* S = scratch_of(ctx);
  MF_TRY(S->a.alloc(sizeof(float) * (size_t)pad * yb));
  MF_TRY(launch_correct_one(&ctx->c, d_proj, nx, ny, shift_x, shift_y, tilt_axis, only_shift, bin,
                            random_fill, S->a.as<float>(), pad, st));
  cufftHandle f, i;
  MF_TRY(ctx->plan({0, xb, yb, yb}, &f));
  MF_TRY(ctx->plan({1, xb, yb, yb}, &i));
  MF_CHECK_CUFFT(cufftExecR2C(f, S->a.as<cufftReal>(), S->a.as<cufftComplex>()));
  MF_TRY(launch_rweight(&ctx->c, S->a.as<cufftComplex>(), cmp, yb, st));
  MF_CHECK_CUFFT(cufftExecC2R(i, S->a.as<cufftComplex>(), d_out));
  return MF_OK;
  MF_GUARD_END
}

MF_API int mf_find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                              int nproj, int* range2) {
  if (!angles || !skip || !range2 || iproj < 0 || iproj >= nz || nproj <= 0)
    return set_error(MF_ERR_ARG, "invalid argument");
  find_proj_range(angles, nz, skip, iproj, nproj, range2);
  return MF_OK;
}

MF_API int mf_dev_reproject(mf_context* ctx, const float* d_corr, int xb, int yb, int nz,
                            const float* angles, int iproj, int istart, int iend, int thickness,
                            int method, float* d_out) {
  MF_GUARD_BEGIN
  MF_TRY(use_device(ctx));
  if (!d_corr || !angles || !d_out) return set_error(MF_ERR_ARG, "null argument");
  if (istart < 0 || iend < istart || iend >= nz || iproj < 0 || iproj >= nz || thickness < 2 ||
      xb < 2 || yb < 1)
    return set_error(MF_ERR_ARG, "invalid re-projection range or size");
  cudaStream_t st = ctx->c.stream;
  ReprojGeom g;
  reproj_geometry(angles, iproj, istart, iend, xb, yb, thickness, &g);
  {
    std::vector<ReprojGeom> gv(1, g);
    MF_TRY(fill_bp_device(&ctx->c, angles, &gv, st));
    g = gv[0];
  }
  mf_context::Scratch* S = scratch_of(ctx);
  MF_TRY(S->b.alloc(sizeof(float) * g.bp.size()));
  MF_CHECK_CUDA(cudaMemcpyAsync(S->b.p, g.bp.data(), sizeof(float) * g.bp.size(),
                                cudaMemcpyHostToDevice, st));
  size_t pix = (size_t)xb * yb;
  if (method == 0) {
    MF_TRY(launch_reproject_exact(&ctx->c, d_corr, xb, yb, pix, S->b.as<float>(), g.i0, g.nk,
                                  g.fcos, g.fsin, g.ray_len, g.thick, nullptr, d_out, st));
  } else if (method == 2 || method == 3) {
    // tensor-core apply on a 16-bit copy of the neighbour tilts
    const int prec = method == 2 ? MF_PREC_FP16 : MF_PREC_BF16;
    const int xpitch = (xb + 7) / 8 * 8;
    const int ytiles = (yb + kApplyTileY - 1) / kApplyTileY;
    TcOpSet set;
    std::vector<ReprojGeom> gs(1, g);
    MF_TRY(build_reproj_tc_ops(&ctx->c, gs, prec, &set, st));
    MF_TRY(S->c.alloc((size_t)2 * xpitch * yb * nz));
    const size_t nflags = (size_t)nz * ytiles * kFlagParts;
    MF_TRY(S->d.alloc(sizeof(int) * (nflags + 1)));
    int* tflags = S->d.as<int>();
    int* err = tflags + nflags;
    MF_CHECK_CUDA(cudaMemsetAsync(S->d.p, 0, sizeof(int) * (nflags + 1), st));
    MF_TRY(launch_to_half(&ctx->c, d_corr, xb, yb, nullptr, istart, iend - istart + 1, prec,
                          S->c.p, xpitch, tflags, st));
    TmaDesc imgmap;
    const int nb = tc_pick_rows(&ctx->c, xb, yb);
    MF_TRY(tc_prepare(&ctx->c, nb));
    MF_TRY(tc_image_map(S->c.p, prec, xb, xpitch, yb, nz, nb, &imgmap));
    MF_TRY(launch_reproject_tc(&ctx->c, set, set.ops[0], imgmap, nb, err, d_out, st));
    MF_TRY(launch_reproject_exact_flagged(&ctx->c, d_corr, xb, yb, pix, S->b.as<float>(), g.i0,
                                          g.nk, g.fcos, g.fsin, g.ray_len, g.thick, tflags, d_out,
                                          st));
    int herr = 0;
    MF_CHECK_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaStreamSynchronize(st));
    if (herr != 0)
      return set_error(MF_ERR_CUDA, "tensor-core re-projection pipeline stalled (code %d)", herr);
  } else {
    ReprojOpSet set;
    std::vector<ReprojGeom> gs(1, g);
    MF_TRY(build_reproj_ops(&ctx->c, gs, &set, st));
    int ytiles = (yb + kApplyTileY - 1) / kApplyTileY;
    MF_TRY(S->c.alloc(sizeof(int) * ytiles));
    MF_CHECK_CUDA(cudaMemsetAsync(S->c.p, 0, sizeof(int) * ytiles, st));
    MF_TRY(launch_reproject_apply(&ctx->c, set.ops[0], d_corr, pix, S->c.as<int>(), d_out, st));
    MF_TRY(launch_reproject_exact(&ctx->c, d_corr, xb, yb, pix, S->b.as<float>(), g.i0, g.nk,
                                  g.fcos, g.fsin, g.ray_len, g.thick, S->c.as<int>(), d_out, st));
  }
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
  MF_GUARD_END
}

MF_API int mf_dev_measure_shift(mf_context* ctx, const float* d_reproj, const float* d_proj,
                                int xb, int yb, float* shift2, float* peak) {
  MF_GUARD_BEGIN
  MF_TRY(use_device(ctx));
  if (!d_reproj || !d_proj || !shift2 || xb < 8 || yb < 8 || (xb & 1))
    return set_error(MF_ERR_ARG, "invalid argument");
  cudaStream_t st = ctx->c.stream;
  const int pad = (xb / 2 + 1) * 2, cmp = pad / 2;
  const size_t ppix = (size_t)pad * yb;
  mf_context::Scratch* S = scratch_of(ctx);
  MF_TRY(S->a.alloc(sizeof(float) * ppix * 2));
  const int mparts = moment_parts(yb) * 2;
  MF_TRY(S->d.alloc(sizeof(double2) * mparts + sizeof(float2) * (kPeakParts + 2) + 64));
  double2* mpart = S->d.as<double2>();
  float2* stats = reinterpret_cast<float2*>(mpart + mparts);
  float2* ppart = stats + 2;
  float* outv = reinterpret_cast<float*>(ppart + kPeakParts);
  float* cc = S->a.as<float>();
  const float mcx = (float)((pad / 2 - 1) * 2) * 0.5f, mcy = (float)yb * 0.5f;
  MF_TRY(norm_mask_pad(&ctx->c, d_reproj, d_proj, xb, 0, xb, yb, pad, ppix, 2, 0, mcx, mcy,
                       (float)pad, (float)yb, 4.0f, nullptr, cc, mpart, stats, st));
  cufftHandle f, i;
  MF_TRY(ctx->plan({2, xb, yb, 2}, &f));
  MF_TRY(ctx->plan({3, xb, yb, 1}, &i));
  MF_CHECK_CUFFT(cufftExecR2C(f, cc, (cufftComplex*)cc));
  MF_TRY(xcorr_filter(&ctx->c, (cufftComplex*)cc, 0, nullptr, (cufftComplex*)(cc + ppix), 0, 1,
                      cmp, yb, 500.0f, 1.0f, st));
  MF_CHECK_CUFFT(cufftExecC2R(i, (cufftComplex*)(cc + ppix), cc + ppix));
  MF_TRY(pa_peak_only(&ctx->c, cc + ppix, pad, xb, yb, ppart, outv, st));
  float h[3];
  MF_CHECK_CUDA(cudaMemcpyAsync(h, outv, sizeof(h), cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  shift2[0] = h[0];
  shift2[1] = h[1];
  if (peak) *peak = h[2];
  return MF_OK;
  MF_GUARD_END
}

}  // extern "C"

