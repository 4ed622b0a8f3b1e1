// Stack correction and pre-processing kernels.
//
// Reference: Markerfree/src/method/CorrStack.cu (mGCorrect + mGRandom :116-179,
// mGBinImage :40-63, GRWeight :431-446) and Markerfree/src/method/Preprocess.cu.
// The reference resamples into a padded buffer, bins it in a second kernel,
// R-weights it with batched 1-D cuFFTs and un-pads it with one cudaMemcpy per
// row.  Here resampling and binning are one kernel that writes straight into the
// row layout the FFT wants, and the inverse FFT writes the dense corrected stack.
#include <algorithm>

#include "mf_internal.hpp"

namespace mf {

// Where pixel (ix, iy) of an in_x x in_y image sits: ix * xs + iy * ys.  The
// row-major stack has (xs, ys) = (1, in_x); its column-major copy (in_y, 1).
struct Layout {
  int xs, ys;
  __device__ __forceinline__ size_t at(int ix, int iy) const {
    return (size_t)ix * xs + (size_t)iy * ys;
  }
};

// Neighbouring output pixels of a row sample the source one step of (cos, sin)
// apart: along a source row when |cos| >= |sin|, else along a source column, which
// the column-major copy (when there is one) holds contiguously.  Both layouts hold
// the same values, so the choice changes addresses only.
__device__ __forceinline__ Layout pick_layout(const float* stack_t, int in_x, int in_y, float cs,
                                              float sn) {
  if (stack_t != nullptr && fabsf(sn) > fabsf(cs)) return Layout{in_y, 1};
  return Layout{1, in_x};
}

// CorrStack.cu:116-140
__device__ __forceinline__ float corr_random(int x, int y, int in_x, int in_y,
                                             const float* __restrict__ img, Layout L) {
  if (x < 0) x = -x;
  if (y < 0) y = -y;
  if (x >= in_x) x = in_x - 1 - (x % in_x);
  if (y >= in_y) y = in_y - 1 - (y % in_y);
  const int win = 51, size = win * win;
  unsigned int next = (unsigned int)(y * in_x + x);
  for (int i = 0; i < 20; ++i) {
    next = (next * 19u + 57u) % (unsigned int)size;
    int ix = (int)(next % (unsigned int)size) - win / 2 + x;
    if (ix < 0 || ix >= in_x) continue;
    int iy = (int)(next / (unsigned int)win) - win / 2 + y;
    if (iy < 0 || iy >= in_y) continue;
    return __ldg(img + L.at(ix, iy));
  }
  return __ldg(img + L.at(x, y));
}

// CorrStack.cu:151-179 for one resampled pixel (X, Y) of an out_x x in_y grid.
__device__ __forceinline__ float corr_pixel(const float* __restrict__ img, Layout L, int in_x,
                                            int in_y, int X, int Y, int out_x, float sx, float sy,
                                            float cs, float sn, bool random_fill) {
  float ax = __fsub_rn(__fadd_rn((float)X, 0.5f), __fmul_rn((float)out_x, 0.5f));
  float ay = __fsub_rn(__fadd_rn((float)Y, 0.5f), __fmul_rn((float)in_y, 0.5f));
  // mGCorrect's rotation as nvcc compiles it: the first product of each sum fused
  float t = __fmaf_rn(ax, cs, -__fmul_rn(ay, sn));
  ay = __fmaf_rn(ax, sn, __fmul_rn(ay, cs));
  ax = t;
  ax = __fadd_rn(ax, __fadd_rn(sx, __fmul_rn((float)in_x, 0.5f)));
  ay = __fadd_rn(ay, __fadd_rn(sy, __fmul_rn((float)in_y, 0.5f)));
  int ix = (int)__fadd_rn(ax, 0.5f);
  int iy = (int)__fadd_rn(ay, 0.5f);
  if (ix >= 0 && ix < in_x && iy >= 0 && iy < in_y) return __ldg(img + L.at(ix, iy));
  if (random_fill) return corr_random(ix, iy, in_x, in_y, img, L);
  return kSentinel;
}

struct CorrArgs {
  const float* stack;
  const float* stack_t;  // column-major copy of the stack, or null
  int nx, ny;
  size_t pix;
  const int* tilts;  // tilt index per blockIdx.z (nullptr: blockIdx.z itself)
  const float* sx;
  const float* sy;
  const float* rot;
  float one_sx, one_sy, one_rot;  // used when sx == nullptr
  int only_shift, bin, random_fill;
  int out_x, xb, yb, binx, biny;
  float* out;
  int out_row_stride;
  size_t out_tilt_stride;
};

__global__ void k_correct_bin(CorrArgs a) {
  __shared__ float s_cs, s_sn, s_sx, s_sy;
  const int j = blockIdx.z;
  const int z = a.tilts ? a.tilts[j] : j;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    float rot = a.sx ? a.rot[z] : a.one_rot;
    float axis = a.only_shift ? 0.0f : rot;
    axis = (float)((double)axis * kD2R);  // CorrStack.cu:376-378
    s_cs = cosf(axis);  // CUDA's cosf/sinf, as mGCorrect (CorrStack.cu:160-161)
    s_sn = sinf(axis);
    s_sx = a.sx ? a.sx[z] : a.one_sx;
    s_sy = a.sx ? a.sy[z] : a.one_sy;
  }
  __syncthreads();
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= a.xb) return;
  const Layout L = pick_layout(a.stack_t, a.nx, a.ny, s_cs, s_sn);
  const float* img = (L.xs == 1 ? a.stack : a.stack_t) + (size_t)z * a.pix;
  // rows in a grid-stride loop: the set-up above is paid once per block
  for (int by = blockIdx.y * blockDim.y + threadIdx.y; by < a.yb; by += gridDim.y * blockDim.y) {
    float res;
    if (a.bin == 1) {
      res = corr_pixel(img, L, a.nx, a.ny, bx, by, a.out_x, s_sx, s_sy, s_cs, s_sn,
                       a.random_fill);
    } else {
      // every sample of the bin is fetched (independent loads); a sentinel among
      // them makes the result the sentinel, as the reference's early exit does
      float sum = 0.0f;
      bool bad = false;
      for (int iy = 0; iy < a.biny; ++iy) {
#pragma unroll 2
        for (int ix = 0; ix < a.binx; ++ix) {
          float v = corr_pixel(img, L, a.nx, a.ny, bx * a.binx + ix, by * a.biny + iy, a.out_x,
                               s_sx, s_sy, s_cs, s_sn, a.random_fill);
          bad |= v < -1e10f;
          sum = __fadd_rn(sum, v);
        }
      }
      res = bad ? kSentinel : sum;
    }
    a.out[(size_t)j * a.out_tilt_stride + (size_t)by * a.out_row_stride + bx] = res;
  }
}

// k_correct_bin for a group of series: job j is tilt (j % nz) of series j / nz,
// or, with a step table, the held-out tilt of series j at that step.
__global__ void k_correct_group(GroupCorrArgs g) {
  __shared__ float s_cs, s_sn, s_sx, s_sy;
  const int j = blockIdx.z;
  const int b = g.steps ? j : j / g.nz_max;
  if (g.active && g.active[b] == 0) return;
  const GroupSeriesDev& S = g.ser[b];
  const int z = g.steps ? g.steps[b].ip : j % g.nz_max;
  if (z < 0 || z >= S.nz) return;  // no held-out tilt at this step / beyond this series
  if ((int)(blockIdx.x * blockDim.x) >= S.xb) return;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const float axis = (float)((double)S.rot[z] * kD2R);  // CorrStack.cu:376-378
    s_cs = cosf(axis);  // CUDA's cosf/sinf, as mGCorrect (CorrStack.cu:160-161)
    s_sn = sinf(axis);
    s_sx = S.sx[z];
    s_sy = S.sy[z];
  }
  __syncthreads();
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= S.xb) return;
  const int nx = S.nx, ny = S.ny, binx = S.binx, biny = S.biny;
  const Layout L = pick_layout(S.stack_t, nx, ny, s_cs, s_sn);
  const float* img = (L.xs == 1 ? S.stack : S.stack_t) + (size_t)z * nx * ny;
  float* out = g.steps ? S.recorr : S.scratch + (size_t)z * S.ppix;
  // rows in a grid-stride loop: the set-up above is paid once per block
  const int step = gridDim.y * blockDim.y;
  int by0 = blockIdx.y * blockDim.y + threadIdx.y;
  if (S.bin == 1) {
    // four rows' gathers in flight before their stores
    for (; by0 + 3 * step < S.yb; by0 += 4 * step) {
      float r[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        r[q] = corr_pixel(img, L, nx, ny, bx, by0 + q * step, S.out_x, s_sx, s_sy, s_cs, s_sn,
                          g.random_fill);
#pragma unroll
      for (int q = 0; q < 4; ++q) out[(size_t)(by0 + q * step) * S.pad + bx] = r[q];
    }
  }
  for (int by = by0; by < S.yb; by += step) {
    float res;
    if (S.bin == 1) {
      res = corr_pixel(img, L, nx, ny, bx, by, S.out_x, s_sx, s_sy, s_cs, s_sn, g.random_fill);
    } else {
      // every sample of the bin is fetched (independent loads); a sentinel among
      // them makes the result the sentinel, as the reference's early exit does
      float sum = 0.0f;
      bool bad = false;
      for (int iy = 0; iy < biny; ++iy) {
#pragma unroll 2
        for (int ix = 0; ix < binx; ++ix) {
          float v = corr_pixel(img, L, nx, ny, bx * binx + ix, by * biny + iy, S.out_x, s_sx,
                               s_sy, s_cs, s_sn, g.random_fill);
          bad |= v < -1e10f;
          sum = __fadd_rn(sum, v);
        }
      }
      res = bad ? kSentinel : sum;
    }
    out[(size_t)by * S.pad + bx] = res;
  }
}

// Row blocks of a resampling launch: each block walks about 16 of its row
// groups, so the per-block set-up (parameter loads, cosf/sinf) is amortised.
static int corr_row_blocks(int rows, int rows_per_block) {
  const int groups = (rows + rows_per_block - 1) / rows_per_block;
  return std::max(1, (groups + 15) / 16);
}

static void fill_sizes(CorrArgs* a, int nx, int ny, int bin) {
  int pad_x = (nx / 2 + 1) * 2;
  a->out_x = (pad_x / 2 - 1) * 2;  // CorrStack.cu:204
  a->xb = nx / bin / 2 * 2;        // CorrStack.cu:72-73
  a->yb = ny / bin / 2 * 2;
  a->binx = a->out_x / a->xb;  // CorrStack.cu:99-100
  a->biny = ny / a->yb;
}

int launch_correct_bin(Context* c, const float* stack, const float* stack_t, int nx, int ny,
                       const int* d_tilts, int ntilts, const float* d_sx, const float* d_sy,
                       const float* d_rot, int only_shift, int bin, int random_fill, float* out,
                       int out_row_stride, size_t out_tilt_stride, cudaStream_t st) {
  CorrArgs a{};
  a.stack = stack;
  a.stack_t = stack_t;
  a.nx = nx;
  a.ny = ny;
  a.pix = (size_t)nx * ny;
  a.tilts = d_tilts;
  a.sx = d_sx;
  a.sy = d_sy;
  a.rot = d_rot;
  a.only_shift = only_shift;
  a.bin = bin;
  a.random_fill = random_fill;
  fill_sizes(&a, nx, ny, bin);
  a.out = out;
  a.out_row_stride = out_row_stride;
  a.out_tilt_stride = out_tilt_stride;
  dim3 blk(32, 8), grd((a.xb + 31) / 32, corr_row_blocks(a.yb, 8), ntilts);
  k_correct_bin<<<grd, blk, 0, st>>>(a);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int launch_correct_group(Context* c, const GroupCorrArgs& g, int nseries, int xb_max, int yb_max,
                         cudaStream_t st) {
  const int njobs = g.steps ? nseries : nseries * g.nz_max;
  dim3 blk(64, 4), grd((xb_max + 63) / 64, corr_row_blocks(yb_max, 4), njobs);
  k_correct_group<<<grd, blk, 0, st>>>(g);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int launch_correct_one(Context* c, const float* img, int nx, int ny, float sx, float sy,
                       float axis_deg, int only_shift, int bin, int random_fill, float* out,
                       int out_row_stride, cudaStream_t st) {
  CorrArgs a{};
  a.stack = img;
  a.nx = nx;
  a.ny = ny;
  a.pix = (size_t)nx * ny;
  a.one_sx = sx;
  a.one_sy = sy;
  a.one_rot = axis_deg;
  a.only_shift = only_shift;
  a.bin = bin;
  a.random_fill = random_fill;
  fill_sizes(&a, nx, ny, bin);
  a.out = out;
  a.out_row_stride = out_row_stride;
  a.out_tilt_stride = 0;
  dim3 blk(32, 8), grd((a.xb + 31) / 32, corr_row_blocks(a.yb, 8), 1);
  k_correct_bin<<<grd, blk, 0, st>>>(a);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// CorrStack.cu:431-446: spectrum / N times 2r (0.55 + 0.45 cos 2 pi r), r = k / N.
// Rows are visited with a grid-stride loop, so any number of rows (a whole group
// of stacks) fits in one launch.
__global__ void k_rweight(cufftComplex* spec, int cmp, int rows) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= cmp) return;
  float fN = 2 * ((float)cmp - 1.0f);
  float r = __fdiv_rn((float)x, fN);
  // CUDA's cosf and the contraction of 0.55f + 0.45f * cosf(...), as in GRWeight
  float cw = cosf(__fmul_rn(6.2831852f, r));
  r = __fmul_rn(__fmul_rn(2.0f, r), __fmaf_rn(0.45f, cw, 0.55f));
  for (int row = blockIdx.y * blockDim.y + threadIdx.y; row < rows;
       row += gridDim.y * blockDim.y) {
    size_t i = (size_t)row * cmp + x;
    cufftComplex v = spec[i];
    v.x = __fdiv_rn(v.x, fN);
    v.y = __fdiv_rn(v.y, fN);
    v.x = __fmul_rn(v.x, r);
    v.y = __fmul_rn(v.y, r);
    spec[i] = v;
  }
}

int launch_rweight(Context* c, cufftComplex* spec, int cmp, int rows, cudaStream_t st) {
  dim3 blk(128, 2), grd((cmp + 127) / 128, std::min((rows + 1) / 2, 16384));
  k_rweight<<<grd, blk, 0, st>>>(spec, cmp, rows);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Group form: blockIdx.z = series; the rows of its scratch (all tilts, steps ==
// null) or of its re-corrected held-out tilt, with its own spectrum width.
__global__ void k_rweight_group(const GroupSeriesDev* __restrict__ ser,
                                const GroupStepDev* __restrict__ steps,
                                const int* __restrict__ active) {
  const int b = blockIdx.z;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  if (steps && steps[b].ip < 0) return;
  const int cmp = S.cmp;
  const int rows = steps ? S.yb : S.nz * S.yb;
  cufftComplex* spec = reinterpret_cast<cufftComplex*>(steps ? S.recorr : S.scratch);
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= cmp) return;
  float fN = 2 * ((float)cmp - 1.0f);
  float r = __fdiv_rn((float)x, fN);
  float cw = cosf(__fmul_rn(6.2831852f, r));
  r = __fmul_rn(__fmul_rn(2.0f, r), __fmaf_rn(0.45f, cw, 0.55f));
  // four rows' loads in flight before their stores (the spectrum is updated in place)
  const int step = gridDim.y * blockDim.y;
  for (int row = blockIdx.y * blockDim.y + threadIdx.y; row < rows; row += 4 * step) {
    cufftComplex v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (row + q * step < rows) v[q] = spec[(size_t)(row + q * step) * cmp + x];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (row + q * step < rows) {
        v[q].x = __fmul_rn(__fdiv_rn(v[q].x, fN), r);
        v[q].y = __fmul_rn(__fdiv_rn(v[q].y, fN), r);
        spec[(size_t)(row + q * step) * cmp + x] = v[q];
      }
  }
}

int launch_rweight_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                         const int* active, int nseries, int cmp_max, int rows_max,
                         cudaStream_t st) {
  // about eight rows per thread
  dim3 blk(128, 2), grd((cmp_max + 127) / 128, std::min((rows_max + 15) / 16, 16384), nseries);
  k_rweight_group<<<grd, blk, 0, st>>>(ser, steps, active);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Pre-processing (Preprocess.cu:103-250).
// Per-block minimum over valid pixels of a range of slices.
__global__ void k_block_min(const float* __restrict__ p, size_t n, float* __restrict__ part) {
  __shared__ float s[256];
  float m = 1e20f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float v = p[i];
    if (v < -1e10f) continue;
    m = fminf(m, v);
  }
  s[threadIdx.x] = m;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) s[threadIdx.x] = fminf(s[threadIdx.x], s[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// SetPositive's stack minimum (fStackMin starts at 1e30, slice minima at 1e20)
// from the block minima: mm[0] = min(1e30, minima...) capped at 1e20.
__global__ void k_min_final(const float* __restrict__ part, int nb, float* __restrict__ mm) {
  __shared__ float s[256];
  float m = 1e30f;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) m = fminf(m, part[i]);
  s[threadIdx.x] = m;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) s[threadIdx.x] = fminf(s[threadIdx.x], s[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) mm[0] = s[0] > 1e20f ? 1e20f : s[0];
}

// One block per slice: FP64 sum and count of (v - min) over the central box; the
// minimum is subtracted only when it is below zero (Preprocess.cu:103-160).
// Each slice's central box is split into kBoxParts bands of rows, one block each;
// FP64 partial sums, added in order by k_mass_scale.
constexpr int kBoxParts = 32;

__global__ void k_box_mean(const float* __restrict__ stack, int nx, int ny,
                           const float* __restrict__ mm, double* __restrict__ sums,
                           int* __restrict__ counts) {
  __shared__ double s_sum[256];
  __shared__ int s_cnt[256];
  const float sub = mm[0];
  const bool subtract = !(sub >= 0);
  const int z = blockIdx.x;
  const int x0 = nx * 1 / 6, y0 = ny * 1 / 6, w = nx * 4 / 6, h = ny * 4 / 6;
  const int ya = h * (int)blockIdx.y / kBoxParts, yz = h * ((int)blockIdx.y + 1) / kBoxParts;
  const float* f = stack + (size_t)z * nx * ny;
  double acc = 0.0;
  int cnt = 0;
  for (int y = ya; y < yz; ++y) {
    const float* row = f + (size_t)(y + y0) * nx + x0;
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
      float v = row[x];
      if (subtract && !(v < -1e10f)) v = __fsub_rn(v, sub);
      if (v <= -1e20f) continue;
      acc += v;
      cnt++;
    }
  }
  s_sum[threadIdx.x] = acc;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
    if (threadIdx.x < hh) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + hh];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + hh];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[(size_t)z * kBoxParts + blockIdx.y] = s_sum[0];
    counts[(size_t)z * kBoxParts + blockIdx.y] = s_cnt[0];
  }
}

// MassNormalization's factors (Preprocess.cu:162-250): every slice is scaled to the
// mean of the zero tilt (file order index `zero`), capped at 1000.
__device__ __forceinline__ float box_mean_of(const double* sums, const int* counts, int z) {
  double s = 0.0;
  long long n = 0;
  for (int b = 0; b < kBoxParts; ++b) {
    s += sums[(size_t)z * kBoxParts + b];
    n += counts[(size_t)z * kBoxParts + b];
  }
  return n == 0 ? 0.0f : (float)(s / (double)n);
}

__global__ void k_mass_scale(const double* __restrict__ sums, const int* __restrict__ counts,
                             int nz, int zero, float* __restrict__ scale) {
  const float ref0 = box_mean_of(sums, counts, zero);
  const float ref = ref0 > 1000.0f ? 1000.0f : ref0;
  for (int i = threadIdx.x; i < nz; i += blockDim.x) {
    const float mean = box_mean_of(sums, counts, i);
    scale[i] = __fdiv_rn(ref, __fadd_rn(mean, 0.00001f));
  }
}

// out = (v - min) * scale[z], skipping sentinels as Subtract and mScale do.
__global__ void k_positive_scale(float* __restrict__ stack, size_t pix, int nz,
                                 const float* __restrict__ mm, const float* __restrict__ scale) {
  const float sub = mm[0];
  const bool subtract = !(sub >= 0);
  size_t n = pix * nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float v = stack[i];
    if (subtract && !(v < -1e10f)) v = __fsub_rn(v, sub);
    if (!(v <= -1e20f)) v = __fmul_rn(v, scale[i / pix]);
    stack[i] = v;
  }
}

// The whole pre-processing is queued on st with no host round trip: the minimum,
// the slice means and the scale factors stay in device memory.
int preprocess_device(Context* c, float* d_stack, int nx, int ny, int nz,
                      const float* file_angles, cudaStream_t st) {
  size_t pix = (size_t)nx * ny;
  size_t n = pix * nz;
  const int nb = 1024;
  DevBuf part, sums, counts, scale, mm;
  MF_TRY(part.alloc(sizeof(float) * nb));
  MF_TRY(sums.alloc(sizeof(double) * nz * kBoxParts));
  MF_TRY(counts.alloc(sizeof(int) * nz * kBoxParts));
  MF_TRY(scale.alloc(sizeof(float) * nz));
  MF_TRY(mm.alloc(sizeof(float)));
  k_block_min<<<nb, 256, 0, st>>>(d_stack, n, part.as<float>());
  k_min_final<<<1, 256, 0, st>>>(part.as<float>(), nb, mm.as<float>());
  k_box_mean<<<dim3(nz, kBoxParts), 256, 0, st>>>(d_stack, nx, ny, mm.as<float>(),
                                                    sums.as<double>(), counts.as<int>());
  // the zero tilt is looked up in the file-order angles (Preprocess.cu:168)
  const int zero = frame_idx_from_tilt(nz, file_angles, 0.0f);
  k_mass_scale<<<1, 256, 0, st>>>(sums.as<double>(), counts.as<int>(), nz, zero,
                                  scale.as<float>());
  k_positive_scale<<<c->sm_count * 8, 256, 0, st>>>(d_stack, pix, nz, mm.as<float>(),
                                                     scale.as<float>());
  c->launches += 5;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

}  // namespace mf
