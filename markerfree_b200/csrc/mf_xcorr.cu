// Cross-correlation kernels around cuFFT: normalise/mask/pad, spectrum filter,
// peak search with sub-pixel fit, and the per-tilt parameter update.
//
// Reference: Markerfree/src/method/CalcCC.cu (GSum2D/GSum1D :48-92, GConv,
// GWiener, GCenterOrigin :95-135, GNormalize :137-147, GStretchRandom :149-171,
// GRoundEdge :173-195, FindPeak :381-435) and ProjAlign.cpp (PANorm :295-312,
// PAFindPeak :325-375, ClacAlignProj :181-241, FitRotCenterZ/RemoveOffsetZ
// :459-501).  The reference copies every cross-correlation map to the host and
// scans it on one CPU thread; here the arg-max, the parabolic fit and the
// parameter update run on the GPU and nothing leaves the device.
#include "mf_internal.hpp"
#include "mf_xcorr.hpp"

namespace mf {

constexpr int kMomRows = 8;  // image rows per partial-sum block

__device__ __forceinline__ const float* image_ptr(const float* src0, const float* src1,
                                                  size_t img_stride, int img) {
  return (img == 1 && src1) ? src1 : src0 + (size_t)img * img_stride;
}

// Source images of a group step: image 2b is series b's re-projection, image
// 2b+1 its held-out projection; series with active[b] == 0 are skipped.
struct ImgTable {
  const float* const* ptrs;  // null: image_ptr() addressing
  const int* active;
};
__device__ __forceinline__ const float* table_ptr(const ImgTable& t, const float* src0,
                                                  const float* src1, size_t img_stride, int img) {
  return t.ptrs ? t.ptrs[img] : image_ptr(src0, src1, img_stride, img);
}
__device__ __forceinline__ bool table_skip(const ImgTable& t, int img) {
  return t.active != nullptr && t.active[img >> 1] == 0;
}

// Block-wide sum of two doubles over 256 threads in a fixed order.
__device__ __forceinline__ double2 block_sum2(double a, double b) {
  __shared__ double s1[8], s2[8];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    s1[w] = a;
    s2[w] = b;
  }
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      r.x += s1[i];
      r.y += s2[i];
    }
  return r;
}

// Masked moments: part[img][blk] = (sum v, sum v^2) over the valid pixels of
// kMomRows rows.  Image 1 is read from src1 when it is given.  Rows and images
// start on 8-byte boundaries (even widths and strides), so each thread reads
// column pairs, the kMomRows rows of a pair all in flight before it adds them.
__device__ __forceinline__ void moment_add(float v, double* a, double* b) {
  const bool ok = !(v < -1e10f);  // sentinels are skipped
  *a += ok ? (double)v : 0.0;
  *b += ok ? (double)__fmul_rn(v, v) : 0.0;
}
__global__ void __launch_bounds__(256) k_moments(const float* __restrict__ src0,
                                                 const float* __restrict__ src1, int w, int h,
                                                 int stride, size_t img_stride,
                                                 double2* __restrict__ part, ImgTable tab) {
  if (table_skip(tab, blockIdx.y)) return;
  const float* p = table_ptr(tab, src0, src1, img_stride, blockIdx.y);
  double a = 0.0, b = 0.0;
  const int y0 = blockIdx.x * kMomRows, nrows = min(h - y0, kMomRows);
  const int npair = w >> 1;
  for (int q = threadIdx.x; q < npair; q += blockDim.x) {
    float2 v[kMomRows];
#pragma unroll
    for (int k = 0; k < kMomRows; ++k)
      v[k] = k < nrows ? __ldg(reinterpret_cast<const float2*>(p + (size_t)(y0 + k) * stride) + q)
                       : make_float2(-1e30f, -1e30f);
#pragma unroll
    for (int k = 0; k < kMomRows; ++k) {
      moment_add(v[k].x, &a, &b);
      moment_add(v[k].y, &a, &b);
    }
  }
  if ((w & 1) && threadIdx.x == 0)  // an odd last column
    for (int k = 0; k < nrows; ++k)
      moment_add(__ldg(p + (size_t)(y0 + k) * stride + w - 1), &a, &b);
  double2 s = block_sum2(a, b);
  if (threadIdx.x == 0) part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// stats[img] = (mean, std).  with_std = 0: std = 1 (PANorm); 1: CalcCC::mNormalize.
__global__ void __launch_bounds__(256) k_moments_final(const double2* __restrict__ part, int nblk,
                                                       int w, int h, int with_std,
                                                       float2* __restrict__ stats) {
  const double2* p = part + (size_t)blockIdx.x * nblk;
  double a0 = 0.0, b0 = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    a0 += p[i].x;
    b0 += p[i].y;
  }
  double2 s = block_sum2(a0, b0);
  if (threadIdx.x != 0) return;
  double a = s.x, b = s.y;
  double n = (double)w * (double)h;
  float mean = (float)(a / n);
  float sd = 1.0f;
  if (with_std) {
    float m2 = (float)(b / n);
    sd = __fsub_rn(m2, __fmul_rn(mean, mean));
    sd = (sd <= 0.0f) ? 0.0f : sqrtf(sd);
  }
  stats[blockIdx.x] = make_float2(mean, sd);
}

// The GRoundEdge factor of pixel (x, y) (CalcCC.cu:173-193) as nvcc compiles it:
// fx*fx + fy*fy contracted, CUDA's cosf; -1 where the reference writes 0.
__device__ __forceinline__ float round_edge(int x, int y, float cx, float cy, float msx,
                                            float msy, float power) {
  float fx = __fdiv_rn(__fmul_rn(2.0f, fabsf(__fsub_rn((float)x, cx))), msx);
  float fy = __fdiv_rn(__fmul_rn(2.0f, fabsf(__fsub_rn((float)y, cy))), msy);
  float fr = sqrtf(__fmaf_rn(fx, fx, __fmul_rn(fy, fy)));
  if (fr >= 1.0f) return -1.0f;
  fr = __fmul_rn(0.5f, __fsub_rn(1.0f, cosf(__fmul_rn(3.1415926f, fr))));
  return __fsub_rn(1.0f, powf(fr, power));
}

// The factor for every pixel of a w x h image: it depends on the geometry only,
// so a projection-matching pass reads it instead of evaluating cosf and powf for
// every pixel of every image.
__global__ void k_round_mask(int w, int h, float cx, float cy, float msx, float msy, float power,
                             float* __restrict__ mask) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x < w && y < h) mask[(size_t)y * w + x] = round_edge(x, y, cx, cy, msx, msy, power);
}

int make_round_mask(Context* c, int w, int h, float cx, float cy, float msx, float msy,
                    float power, float* d_mask, cudaStream_t st) {
  dim3 blk(64, 4), grd((w + 63) / 64, (h + 3) / 4);
  k_round_mask<<<grd, blk, 0, st>>>(w, h, cx, cy, msx, msy, power, d_mask);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Normalise with stats, apply GRoundEdge (from `mask` when given), zero the pad
// columns; reads rows of `src_stride` floats (first w used) and writes rows of
// `pad` floats.
// Each thread takes one column of four consecutive rows, all loads issued first.
__global__ void k_norm_mask(const float* __restrict__ src, const float* __restrict__ src1,
                            int src_stride, size_t src_img_stride, int w, int h, int pad,
                            size_t dst_img_stride, const float2* __restrict__ stats, float cx,
                            float cy, float msx, float msy, float power,
                            const float* __restrict__ mask, float* __restrict__ dst,
                            ImgTable tab) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y0 = (blockIdx.y * blockDim.y + threadIdx.y) * 4;
  int img = blockIdx.z;
  if (x >= pad || y0 >= h || table_skip(tab, img)) return;
  const int nr = min(4, h - y0);
  float* d = dst + (size_t)img * dst_img_stride + (size_t)y0 * pad + x;
  if (x >= w) {
    for (int r = 0; r < nr; ++r) d[(size_t)r * pad] = 0.0f;
    return;
  }
  const float* sp = table_ptr(tab, src, src1, src_img_stride, img) + (size_t)y0 * src_stride + x;
  float v[4], fm[4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (r < nr) {
      v[r] = sp[(size_t)r * src_stride];
      fm[r] = mask ? __ldg(mask + (size_t)(y0 + r) * w + x) : 0.0f;
    }
  const float2 st = stats[img];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (r >= nr) break;
    float vv = v[r];
    if (!(vv < -1e10f)) {  // GNormalize; a division by 1 (PANorm) is exact and skipped
      vv = __fsub_rn(vv, st.x);
      if (st.y != 1.0f) vv = __fdiv_rn(vv, st.y);
    }
    if (vv < -1e10f) {  // GRoundEdge
      d[(size_t)r * pad] = 0.0f;
      continue;
    }
    const float fr = mask ? fm[r] : round_edge(x, y0 + r, cx, cy, msx, msy, power);
    d[(size_t)r * pad] = fr < 0.0f ? 0.0f : __fmul_rn(vv, fr);
  }
}

int moment_parts(int h) { return (h + kMomRows - 1) / kMomRows; }

int norm_mask_pad(Context* c, const float* src, const float* src1, int src_stride,
                  size_t src_img_stride, int w, int h, int pad, size_t dst_img_stride, int nimg,
                  int with_std, float cx, float cy, float msx, float msy, float power,
                  const float* mask, float* dst, double2* d_part, float2* d_stats,
                  cudaStream_t st) {
  const int nb = moment_parts(h);
  const ImgTable tab{nullptr, nullptr};
  k_moments<<<dim3(nb, nimg), 256, 0, st>>>(src, src1, w, h, src_stride, src_img_stride, d_part,
                                            tab);
  k_moments_final<<<nimg, 256, 0, st>>>(d_part, nb, w, h, with_std, d_stats);
  dim3 blk(64, 4), grd((pad + 63) / 64, (h + 15) / 16, nimg);
  k_norm_mask<<<grd, blk, 0, st>>>(src, src1, src_stride, src_img_stride, w, h, pad,
                                   dst_img_stride, d_stats, cx, cy, msx, msy, power, mask, dst,
                                   tab);
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Group form of PANorm for one step: image 2b is series b's re-projection, image
// 2b+1 its held-out projection (corr + ip * bpix), each with its series' size,
// mask and buffers; the arithmetic and its order are norm_mask_pad's.
__device__ __forceinline__ const float* group_image(const GroupSeriesDev& S, const GroupStepDev& T,
                                                    int img) {
  return (img & 1) ? S.corr + (size_t)T.ip * S.bpix : S.reproj;
}

__global__ void __launch_bounds__(256) k_moments_group(const GroupSeriesDev* __restrict__ ser,
                                                       const GroupStepDev* __restrict__ steps,
                                                       const int* __restrict__ active) {
  const int img = blockIdx.y, b = img >> 1;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  const GroupStepDev T = steps[b];
  const int nblk = (S.yb + kMomRows - 1) / kMomRows;  // moment_parts(yb)
  if (T.ip < 0 || (int)blockIdx.x >= nblk) return;
  const float* p = group_image(S, T, img);
  const int w = S.xb, h = S.yb;
  double a = 0.0, bb = 0.0;
  const int y0 = blockIdx.x * kMomRows, nrows = min(h - y0, kMomRows);
  const int npair = w >> 1;
  for (int q = threadIdx.x; q < npair; q += blockDim.x) {
    float2 v[kMomRows];
#pragma unroll
    for (int k = 0; k < kMomRows; ++k)
      v[k] = k < nrows ? __ldg(reinterpret_cast<const float2*>(p + (size_t)(y0 + k) * w) + q)
                       : make_float2(-1e30f, -1e30f);
#pragma unroll
    for (int k = 0; k < kMomRows; ++k) {
      moment_add(v[k].x, &a, &bb);
      moment_add(v[k].y, &a, &bb);
    }
  }
  if ((w & 1) && threadIdx.x == 0)
    for (int k = 0; k < nrows; ++k) moment_add(__ldg(p + (size_t)(y0 + k) * w + w - 1), &a, &bb);
  double2 s2 = block_sum2(a, bb);
  if (threadIdx.x == 0) S.mpart[(size_t)(img & 1) * nblk + blockIdx.x] = s2;
}

__global__ void __launch_bounds__(256) k_moments_final_group(
    const GroupSeriesDev* __restrict__ ser, const GroupStepDev* __restrict__ steps,
    const int* __restrict__ active) {
  const int img = blockIdx.x, b = img >> 1;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  if (steps[b].ip < 0) return;
  const int nblk = (S.yb + kMomRows - 1) / kMomRows;  // moment_parts(yb)
  const double2* p = S.mpart + (size_t)(img & 1) * nblk;
  double a0 = 0.0, b0 = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    a0 += p[i].x;
    b0 += p[i].y;
  }
  double2 s2 = block_sum2(a0, b0);
  if (threadIdx.x != 0) return;
  double n = (double)S.xb * (double)S.yb;
  S.stats[img & 1] = make_float2((float)(s2.x / n), 1.0f);  // PANorm: std = 1
}

// Two neighbouring pixels per thread (widths and pitches are even): the image,
// mask and output rows are read and written as float2.
__device__ __forceinline__ float norm_mask_one(float v, float mean, float fr) {
  if (!(v < -1e10f)) v = __fsub_rn(v, mean);  // GNormalize with std 1
  if (v < -1e10f) return 0.0f;
  return fr < 0.0f ? 0.0f : __fmul_rn(v, fr);
}

// Each thread takes a pixel pair in kNmRows consecutive rows and issues all their
// loads before the arithmetic, so that enough bytes are in flight to stream the
// images at memory speed.
constexpr int kNmRows = 4;

__global__ void k_norm_mask_group(const GroupSeriesDev* __restrict__ ser,
                                  const GroupStepDev* __restrict__ steps,
                                  const int* __restrict__ active) {
  const int img = blockIdx.z, b = img >> 1;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  const GroupStepDev T = steps[b];
  if (T.ip < 0) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;  // pixel pair
  const int y0 = (blockIdx.y * blockDim.y + threadIdx.y) * kNmRows;
  const int w = S.xb, pad = S.pad, yb = S.yb;
  if (2 * q >= pad || y0 >= yb) return;
  const int nr = min(kNmRows, yb - y0);
  float2* d = reinterpret_cast<float2*>(S.cc + (size_t)(img & 1) * S.ppix + (size_t)y0 * pad) + q;
  const size_t dstep = pad / 2;  // float2 per output row
  if (2 * q >= w) {
    for (int r = 0; r < nr; ++r) d[r * dstep] = make_float2(0.0f, 0.0f);
    return;
  }
  const float2* src = reinterpret_cast<const float2*>(group_image(S, T, img) + (size_t)y0 * w) + q;
  const float2* msk = reinterpret_cast<const float2*>(S.mask + (size_t)y0 * w) + q;
  const size_t sstep = w / 2;
  float2 v[kNmRows], fr[kNmRows];
#pragma unroll
  for (int r = 0; r < kNmRows; ++r)
    if (r < nr) {
      v[r] = src[r * sstep];
      fr[r] = __ldg(msk + r * sstep);
    }
  const float mean = S.stats[img & 1].x;
#pragma unroll
  for (int r = 0; r < kNmRows; ++r)
    if (r < nr)
      d[r * dstep] = make_float2(norm_mask_one(v[r].x, mean, fr[r].x),
                                 norm_mask_one(v[r].y, mean, fr[r].y));
}

int norm_mask_pad_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                        const int* active, int nseries, int xb_max, int yb_max, int pad_max,
                        cudaStream_t st) {
  (void)xb_max;
  k_moments_group<<<dim3(moment_parts(yb_max), 2 * nseries), 256, 0, st>>>(ser, steps, active);
  k_moments_final_group<<<2 * nseries, 256, 0, st>>>(ser, steps, active);
  dim3 blk(128, 2), grd((pad_max / 2 + 127) / 128, (yb_max + 2 * kNmRows - 1) / (2 * kNmRows),
                        2 * nseries);
  k_norm_mask_group<<<grd, blk, 0, st>>>(ser, steps, active);
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// conj(R) * I, B-factor / amplitude (Wiener-like) filter and origin centring,
// written over I.  `scale` reproduces GMultiplyFactor (1/N after each R2C) when
// != 1.  Pair p uses ref spectrum ref + idx[p]*ref_stride (idx[p] = p when idx is
// null) and image img + p*img_stride.
__global__ void k_xcorr_filter(const cufftComplex* __restrict__ ref, size_t ref_stride,
                               const int* __restrict__ ref_idx, cufftComplex* __restrict__ img,
                               size_t img_stride, int cmp, int ny, float bfactor, float scale) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= cmp || y >= ny) return;
  size_t i = (size_t)y * cmp + x;
  const int ri = ref_idx ? ref_idx[blockIdx.z] : (int)blockIdx.z;
  cufftComplex A = ref[(size_t)ri * ref_stride + i];
  cufftComplex* Bp = img + (size_t)blockIdx.z * img_stride + i;
  cufftComplex B = *Bp;
  if (scale != 1.0f) {
    A.x = __fmul_rn(A.x, scale);
    A.y = __fmul_rn(A.y, scale);
    B.x = __fmul_rn(B.x, scale);
    B.y = __fmul_rn(B.y, scale);
  }
  // GConv + GWiener (CalcCC.cu:95-123) as nvcc compiles them: the first product of
  // each sum of products fused, CUDA's expf
  float re = __fmaf_rn(A.x, B.x, __fmul_rn(A.y, B.y));
  float im = __fmaf_rn(A.x, B.y, -__fmul_rn(A.y, B.x));
  int yy = y;
  if (yy > ny / 2) yy -= ny;
  float fnx = __fmul_rn(2.0f, (float)(cmp - 1));
  float filt = __fdiv_rn(__fmul_rn(-2.0f, bfactor), __fmaf_rn(fnx, fnx, (float)(ny * ny)));
  float k2 = (float)((unsigned)(x * x) + (unsigned)(yy * yy));
  filt = expf(__fmul_rn(filt, k2));
  float amp = sqrtf(__fmaf_rn(re, re, __fmul_rn(im, im)));
  filt = __fdiv_rn(filt, sqrtf(__fadd_rn(amp, 0.01f)));
  re = __fmul_rn(re, filt);
  im = __fmul_rn(im, filt);
  if ((x + y) & 1) {
    re = -re;
    im = -im;
  }
  *Bp = make_cuComplex(re, im);
}

// Group form: blockIdx.z = series; its pair's spectra in its cc buffer.
// Two rows per thread (y and y + ny/2 rounded up), both spectra pairs loaded
// before the arithmetic.
__device__ __forceinline__ cufftComplex xcorr_filter_one(cufftComplex A, cufftComplex B, int x,
                                                         int y, int cmp, int ny, float bfactor) {
  float re = __fmaf_rn(A.x, B.x, __fmul_rn(A.y, B.y));
  float im = __fmaf_rn(A.x, B.y, -__fmul_rn(A.y, B.x));
  int yy = y;
  if (yy > ny / 2) yy -= ny;
  float fnx = __fmul_rn(2.0f, (float)(cmp - 1));
  float filt = __fdiv_rn(__fmul_rn(-2.0f, bfactor), __fmaf_rn(fnx, fnx, (float)(ny * ny)));
  float k2 = (float)((unsigned)(x * x) + (unsigned)(yy * yy));
  filt = expf(__fmul_rn(filt, k2));
  float amp = sqrtf(__fmaf_rn(re, re, __fmul_rn(im, im)));
  filt = __fdiv_rn(filt, sqrtf(__fadd_rn(amp, 0.01f)));
  re = __fmul_rn(re, filt);
  im = __fmul_rn(im, filt);
  if ((x + y) & 1) {
    re = -re;
    im = -im;
  }
  return make_cuComplex(re, im);
}

__global__ void k_xcorr_filter_group(const GroupSeriesDev* __restrict__ ser,
                                     const GroupStepDev* __restrict__ steps,
                                     const int* __restrict__ active, float bfactor) {
  const int b = blockIdx.z;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  if (steps[b].ip < 0) return;
  const int cmp = S.cmp, ny = S.yb, half = (ny + 1) / 2;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y0 = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= cmp || y0 >= half) return;
  const int y1 = y0 + half;
  const bool two = y1 < ny;
  const cufftComplex* Ap = reinterpret_cast<const cufftComplex*>(S.cc);
  cufftComplex* Bp = reinterpret_cast<cufftComplex*>(S.cc + S.ppix);
  const size_t i0 = (size_t)y0 * cmp + x, i1 = (size_t)y1 * cmp + x;
  const cufftComplex A0 = Ap[i0], B0 = Bp[i0];
  cufftComplex A1 = A0, B1 = B0;
  if (two) {
    A1 = Ap[i1];
    B1 = Bp[i1];
  }
  Bp[i0] = xcorr_filter_one(A0, B0, x, y0, cmp, ny, bfactor);
  if (two) Bp[i1] = xcorr_filter_one(A1, B1, x, y1, cmp, ny, bfactor);
}

int xcorr_filter_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                       const int* active, int nseries, int cmp_max, int yb_max, float bfactor,
                       cudaStream_t st) {
  dim3 blk(64, 4), grd((cmp_max + 63) / 64, ((yb_max + 1) / 2 + 3) / 4, nseries);
  k_xcorr_filter_group<<<grd, blk, 0, st>>>(ser, steps, active, bfactor);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int xcorr_filter(Context* c, const cufftComplex* ref, size_t ref_stride, const int* d_ref_idx,
                 cufftComplex* img, size_t img_stride, int npairs, int cmp, int ny, float bfactor,
                 float scale, cudaStream_t st) {
  dim3 blk(64, 4), grd((cmp + 63) / 64, (ny + 3) / 4, npairs);
  k_xcorr_filter<<<grd, blk, 0, st>>>(ref, ref_stride, d_ref_idx, img, img_stride, cmp, ny,
                                      bfactor, scale);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Arg-max over a window [sx, ex) x [sy, ey) of a real map (row stride `stride`).
// Ties go to the smallest row-major index, as in the reference's scan.
__device__ __forceinline__ bool better(float v, int i, float bv, int bi) {
  return v > bv || (v == bv && i < bi);
}

// Each block scans a band of rows of the window (rows split evenly over gridDim.x).
__global__ void __launch_bounds__(256) k_peak_partial(const float* __restrict__ map,
                                                      size_t map_stride, int stride, int sx,
                                                      int ex, int sy, int ey,
                                                      float2* __restrict__ part) {
  __shared__ float sv[256];
  __shared__ int si[256];
  const float* m = map + (size_t)blockIdx.y * map_stride;
  const int rows = ey - sy;
  const int r0 = sy + (int)((long long)rows * blockIdx.x / gridDim.x);
  const int r1 = sy + (int)((long long)rows * (blockIdx.x + 1) / gridDim.x);
  float bv = -INFINITY;
  int bi = INT_MAX;
  for (int y = r0; y < r1; ++y) {
#pragma unroll 4
    for (int x = sx + threadIdx.x; x < ex; x += blockDim.x) {
      int li = y * stride + x;
      float v = __ldg(m + li);
      if (better(v, li, bv, bi)) {
        bv = v;
        bi = li;
      }
    }
  }
  sv[threadIdx.x] = bv;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h && better(sv[threadIdx.x + h], si[threadIdx.x + h], sv[threadIdx.x],
                                  si[threadIdx.x])) {
      sv[threadIdx.x] = sv[threadIdx.x + h];
      si[threadIdx.x] = si[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = make_float2(sv[0], __int_as_float(si[0]));
}

// Called by all 32 lanes of warp 0; every lane gets the winner.
__device__ void reduce_partials(const float2* p, int n, float* bv, int* bi) {
  float v = -INFINITY;
  int idx = INT_MAX;
  for (int i = threadIdx.x; i < n; i += 32) {
    float pv = p[i].x;
    int pi = __float_as_int(p[i].y);
    if (better(pv, pi, v, idx)) {
      v = pv;
      idx = pi;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    float ov = __shfl_xor_sync(0xffffffffu, v, o);
    int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (better(ov, oi, v, idx)) {
      v = ov;
      idx = oi;
    }
  }
  *bv = v;
  *bi = idx;
}

// Integer peak from the reduced linear index.  When no pixel of the window
// compared as a maximum (all NaN) the reference keeps its initial peak (0, 0),
// whose neighbours lie outside the map; the window's first pixel is used instead.
__device__ __forceinline__ void pa_window_peak(int bi, int stride, int xb, int yb, int* px,
                                               int* py) {
  if (bi == INT_MAX) {
    int sx = xb / 20, sy = yb / 20;
    *px = sx < 3 ? 3 : sx;
    *py = sy < 3 ? 3 : sy;
    return;
  }
  *px = bi % stride;
  *py = bi / stride;
}

// ProjAlign.cpp:350-372: parabolic sub-pixel fit (FP64) around the integer peak.
__device__ void pa_fit(const float* m, int stride, int px, int py, double* dx, double* dy,
                       double* peak) {
  int ic = py * stride + px;
  float cxp = m[ic + 1], cxm = m[ic - 1], cyp = m[ic + stride], cym = m[ic - stride],
        cc = m[ic];
  double a = (double)__fadd_rn(cxp, cxm) * 0.5 - (double)cc;
  double b = (double)__fsub_rn(cxp, cxm) * 0.5;
  double c = (double)__fadd_rn(cyp, cym) * 0.5 - (double)cc;
  double d = (double)__fsub_rn(cyp, cym) * 0.5;
  double ddx = -b / (2 * a + 1e-30);
  double ddy = -d / (2 * c + 1e-30);
  if (fabs(ddx) > 1) ddx = 0;
  if (fabs(ddy) > 1) ddy = 0;
  *dx = ddx;
  *dy = ddy;
  *peak = a * ddx * ddx + b * ddx + c * ddy * ddy + d * ddy + (double)cc;
}

__device__ __forceinline__ void rot_shift(float in0, float in1, float angle_deg, float* o0,
                                          float* o1) {
  float c = (float)cos((double)angle_deg * kD2R);
  float s = (float)sin((double)angle_deg * kD2R);
  float sx = __fsub_rn(__fmul_rn(in0, c), __fmul_rn(in1, s));
  float sy = __fadd_rn(__fmul_rn(in0, s), __fmul_rn(in1, c));
  *o0 = sx;
  *o1 = sy;
}

// CalcZInducedShift (ProjAlign.cpp:553-561)
__device__ __forceinline__ void z_induced(float z0, float angle, float rot, float* s0,
                                          float* s1) {
  *s0 = 0.0f;
  *s1 = 0.0f;
  if (z0 == 0.0f) return;
  float t = (float)((double)angle * kD2R);
  float a = (float)(-(double)z0 * sin((double)t));
  rot_shift(a, 0.0f, rot, s0, s1);
}

// Rotation of a shift and the z-induced shift in FP64 (the forms below, for the
// FP64 accumulation of the FP16/BF16 modes).
__device__ __forceinline__ void rot_shift64(double in0, double in1, float angle_deg, double* o0,
                                            double* o1) {
  const double c = cos((double)angle_deg * kD2R), s = sin((double)angle_deg * kD2R);
  *o0 = in0 * c - in1 * s;
  *o1 = in0 * s + in1 * c;
}
__device__ __forceinline__ void z_induced64(float z0, float angle, float rot, double* s0,
                                            double* s1) {
  *s0 = 0.0;
  *s1 = 0.0;
  if (z0 == 0.0f) return;
  rot_shift64(-(double)z0 * sin((double)angle * kD2R), 0.0, rot, s0, s1);
}

// ClacAlignProj (ProjAlign.cpp:181-241) for held-out tilt ip from the integer peak
// (px, py) of the correlation map: sub-pixel fit, binned -> un-binned shift, the
// measured shift printed by the reference, its rotation by the tilt axis plus the
// z-induced shift added to the tilt's shift, and |shift| as the tilt's error.
// With sx64 (FP16/BF16 modes) the update is formed from the FP64 fit in FP64 and
// accumulated there, sx receiving the float value; otherwise every step is the
// reference's float arithmetic.
__device__ void pa_update(const float* map, int stride, int xb, int yb, int px, int py, int ip,
                          int nx, int ny, const float* angles, float* sx, float* sy,
                          double* sx64, double* sy64, const float* rot, float z0, float* err,
                          float* meas) {
  double dx, dy, pk;
  pa_fit(map, stride, px, py, &dx, &dy, &pk);
  const float r = rot[ip];
  if (sx64 != nullptr) {
    const double a0 = ((double)px + dx - (double)(xb / 2)) * ((double)nx / (double)xb);
    const double a1 = ((double)py + dy - (double)(yb / 2)) * ((double)ny / (double)yb);
    if (meas) {
      meas[2 * ip] = (float)a0;
      meas[2 * ip + 1] = (float)a1;
    }
    double b0, b1, i0, i1;
    rot_shift64(a0, a1, r, &b0, &b1);
    z_induced64(z0, angles[ip], r, &i0, &i1);
    sx64[ip] += b0 + i0;
    sy64[ip] += b1 + i1;
    sx[ip] = (float)sx64[ip];
    sy[ip] = (float)sy64[ip];
    err[ip] = (float)sqrt(a0 * a0 + a1 * a1);
    return;
  }
  float pkx = (float)(px + dx), pky = (float)(py + dy);
  float shx = __fsub_rn(pkx, (float)(xb / 2));
  float shy = __fsub_rn(pky, (float)(yb / 2));
  float binx = __fdiv_rn((float)nx, (float)xb), biny = __fdiv_rn((float)ny, (float)yb);
  float a0 = __fmul_rn(shx, binx), a1 = __fmul_rn(shy, biny);
  float fs = __fadd_rn(__fmul_rn(a0, a0), __fmul_rn(a1, a1));
  fs = sqrtf(fs);
  if (meas) {  // the shift the reference prints (ProjAlign.cpp:203)
    meas[2 * ip] = a0;
    meas[2 * ip + 1] = a1;
  }
  rot_shift(a0, a1, r, &a0, &a1);
  float i0, i1;
  z_induced(z0, angles[ip], r, &i0, &i1);
  a0 = __fadd_rn(a0, i0);
  a1 = __fadd_rn(a1, i1);
  sx[ip] = __fadd_rn(sx[ip], a0);
  sy[ip] = __fadd_rn(sy[ip], a1);
  err[ip] = fs;
}

// Final peak + ClacAlignProj update for held-out tilt ip.
__global__ void k_pa_peak_update(const float* __restrict__ map, int stride, int xb, int yb,
                                 const float2* __restrict__ part, int nparts, int ip, int nx,
                                 int ny, const float* __restrict__ angles, float* __restrict__ sx,
                                 float* __restrict__ sy, double* __restrict__ sx64,
                                 double* __restrict__ sy64, const float* __restrict__ rot,
                                 const float* __restrict__ z0p, float* __restrict__ err,
                                 float* __restrict__ meas) {
  float bv;
  int bi;
  reduce_partials(part, nparts, &bv, &bi);
  if (threadIdx.x != 0) return;
  int px = 0, py = 0;
  pa_window_peak(bi, stride, xb, yb, &px, &py);
  pa_update(map, stride, xb, yb, px, py, ip, nx, ny, angles, sx, sy, sx64, sy64, rot, *z0p, err,
            meas);
}

// Group form of the peak search: blockIdx.y = series; its correlation map (the
// second image of its cc buffer), its own search window, partials in its ppart.
__global__ void __launch_bounds__(256) k_peak_partial_group(
    const GroupSeriesDev* __restrict__ ser, const GroupStepDev* __restrict__ steps,
    const int* __restrict__ active) {
  __shared__ float sv[256];
  __shared__ int si[256];
  const int b = blockIdx.y;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  if (steps[b].ip < 0) return;
  const int xb = S.xb, yb = S.yb, stride = S.pad;
  int sx = xb / 20, sy = yb / 20;
  if (sx < 3) sx = 3;
  if (sy < 3) sy = 3;
  const int ex = xb - sx, ey = yb - sy;
  const float* m = S.cc + S.ppix;
  const int rows = ey - sy;
  const int r0 = sy + (int)((long long)rows * blockIdx.x / gridDim.x);
  const int r1 = sy + (int)((long long)rows * (blockIdx.x + 1) / gridDim.x);
  float bv = -INFINITY;
  int bi = INT_MAX;
  // pixel pairs (the pitch is even, so rows start on 8-byte boundaries); the
  // winner is the largest value, ties to the lowest index, whatever the order
  const int p0 = sx >> 1, p1 = (ex + 1) >> 1;
  for (int y = r0; y < r1; ++y) {
    const float2* row = reinterpret_cast<const float2*>(m + (size_t)y * stride);
#pragma unroll 4
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
      const float2 v = __ldg(row + p);
      const int x = 2 * p, li = y * stride + x;
      if (x >= sx && better(v.x, li, bv, bi)) {
        bv = v.x;
        bi = li;
      }
      if (x + 1 < ex && better(v.y, li + 1, bv, bi)) {
        bv = v.y;
        bi = li + 1;
      }
    }
  }
  sv[threadIdx.x] = bv;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h && better(sv[threadIdx.x + h], si[threadIdx.x + h], sv[threadIdx.x],
                                  si[threadIdx.x])) {
      sv[threadIdx.x] = sv[threadIdx.x + h];
      si[threadIdx.x] = si[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) S.ppart[blockIdx.x] = make_float2(sv[0], __int_as_float(si[0]));
}

// Group form of the peak + ClacAlignProj update: blockIdx.x = series b.
__global__ void k_pa_peak_update_group(const GroupSeriesDev* __restrict__ ser,
                                       const GroupStepDev* __restrict__ steps,
                                       const int* __restrict__ active, int nparts) {
  const int b = blockIdx.x;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  const int ip = steps[b].ip;
  if (ip < 0) return;
  float bv;
  int bi;
  reduce_partials(S.ppart, nparts, &bv, &bi);
  if (threadIdx.x != 0) return;
  int px = 0, py = 0;
  pa_window_peak(bi, S.pad, S.xb, S.yb, &px, &py);
  pa_update(S.cc + S.ppix, S.pad, S.xb, S.yb, px, py, ip, S.nx, S.ny, S.angles, S.sx, S.sy,
            S.sx64, S.sy64, S.rot, *S.z0, S.err, S.meas);
}

int pa_peak_update_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                         const int* active, int nseries, cudaStream_t st) {
  const int nb = kPeakParts;
  k_peak_partial_group<<<dim3(nb, nseries), 256, 0, st>>>(ser, steps, active);
  k_pa_peak_update_group<<<nseries, 32, 0, st>>>(ser, steps, active, nb);
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int pa_peak_update(Context* c, const float* map, int stride, int xb, int yb, float2* d_part,
                   int ip, int nx, int ny, const float* d_angles, float* d_sx, float* d_sy,
                   double* d_sx64, double* d_sy64, const float* d_rot, const float* d_z0,
                   float* d_err, float* d_meas, cudaStream_t st) {
  int sx = xb / 20, sy = yb / 20;
  if (sx < 3) sx = 3;
  if (sy < 3) sy = 3;
  int ex = xb - sx, ey = yb - sy;
  const int nb = kPeakParts;
  k_peak_partial<<<dim3(nb, 1), 256, 0, st>>>(map, 0, stride, sx, ex, sy, ey, d_part);
  k_pa_peak_update<<<1, 32, 0, st>>>(map, stride, xb, yb, d_part, nb, ip, nx, ny, d_angles, d_sx,
                                     d_sy, d_sx64, d_sy64, d_rot, d_z0, d_err, d_meas);
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Plain peak (PAFindPeak) returning the binned shift and peak value into out[3].
__global__ void k_pa_peak_only(const float* __restrict__ map, int stride, int xb, int yb,
                               const float2* __restrict__ part, int nparts, float* out) {
  float bv;
  int bi;
  reduce_partials(part, nparts, &bv, &bi);
  if (threadIdx.x != 0) return;
  int px, py;
  pa_window_peak(bi, stride, xb, yb, &px, &py);
  double dx, dy, pk;
  pa_fit(map, stride, px, py, &dx, &dy, &pk);
  out[0] = __fsub_rn((float)(px + dx), (float)(xb / 2));
  out[1] = __fsub_rn((float)(py + dy), (float)(yb / 2));
  out[2] = (float)pk;
}

int pa_peak_only(Context* c, const float* map, int stride, int xb, int yb, float2* d_part,
                 float* d_out, cudaStream_t st) {
  int sx = xb / 20, sy = yb / 20;
  if (sx < 3) sx = 3;
  if (sy < 3) sy = 3;
  const int nb = kPeakParts;
  k_peak_partial<<<dim3(nb, 1), 256, 0, st>>>(map, 0, stride, sx, xb - sx, sy, yb - sy, d_part);
  k_pa_peak_only<<<1, 32, 0, st>>>(map, stride, xb, yb, d_part, nb, d_out);
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// CalcCC::FindPeak (CalcCC.cu:381-435) for many maps: central 80% window, peak
// clamped to [1, w-2] x [1, h-2], fit in float-promoted arithmetic.
__global__ void k_cc_peak_final(const float* __restrict__ maps, size_t map_stride, int stride,
                                int w, int h, const float2* __restrict__ part, int nparts,
                                float2* __restrict__ shifts) {
  const float* m = maps + (size_t)blockIdx.x * map_stride;
  float bv;
  int bi;
  reduce_partials(part + (size_t)blockIdx.x * nparts, nparts, &bv, &bi);
  if (threadIdx.x != 0) return;
  int px = 0, py = 0;
  if (bi != INT_MAX) {
    px = bi % stride;
    py = bi / stride;
  }
  if (px < 1)
    px = 1;
  else if (px > w - 2)
    px = w - 2;
  if (py < 1)
    py = 1;
  else if (py > h - 2)
    py = h - 2;
  int ic = py * stride + px;
  float cc = m[ic];
  double a = (double)__fsub_rn(__fmul_rn(__fadd_rn(m[ic + 1], m[ic - 1]), 0.5f), cc);
  double b = (double)__fmul_rn(__fsub_rn(m[ic + 1], m[ic - 1]), 0.5f);
  double c = (double)__fsub_rn(__fmul_rn(__fadd_rn(m[ic + stride], m[ic - stride]), 0.5f), cc);
  double d = (double)__fmul_rn(__fsub_rn(m[ic + stride], m[ic - stride]), 0.5f);
  double dx = -b / (2 * a + 1e-30), dy = -d / (2 * c + 1e-30);
  if (fabs(dx) > 1) dx = 0;
  if (fabs(dy) > 1) dy = 0;
  shifts[blockIdx.x] = make_float2(__fsub_rn((float)(px + dx), (float)(w / 2)),
                                   __fsub_rn((float)(py + dy), (float)(h / 2)));
}

int cc_peaks(Context* c, const float* maps, size_t map_stride, int stride, int w, int h, int nmaps,
             float2* d_part, float2* d_shifts, cudaStream_t st) {
  int ssx = w * 8 / 20 * 2, ssy = h * 8 / 20 * 2;
  int sx = (w - ssx) / 2, sy = (h - ssy) / 2;
  const int nb = 32;
  k_peak_partial<<<dim3(nb, nmaps), 256, 0, st>>>(maps, map_stride, stride, sx, sx + ssx, sy,
                                                  sy + ssy, d_part);
  k_cc_peak_final<<<nmaps, 32, 0, st>>>(maps, map_stride, stride, w, h, d_part, nb, d_shifts);
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// FitRotCenterZ + RemoveOffsetZ(-1) (ProjAlign.cpp:459-501, 553-579); the
// reference's uninitialised accumulator dA is taken as 0.  With sx64/sy64 (FP16/BF16
// modes) the shifts are read from and the z-induced shifts removed in FP64.
__device__ void fit_z0_one(int nz, int zt, const float* __restrict__ angles, float* sx,
                           float* sy, double* sx64, double* sy64, const float* __restrict__ rot,
                           float* z0p);

__global__ void k_fit_z0(int nz, int zt, const float* __restrict__ angles, float* sx, float* sy,
                         double* sx64, double* sy64, const float* __restrict__ rot, float* z0p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  fit_z0_one(nz, zt, angles, sx, sy, sx64, sy64, rot, z0p);
}

__global__ void k_fit_z0_group(const GroupSeriesDev* __restrict__ ser,
                               const int* __restrict__ active) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0 || (active && active[b] == 0)) return;
  const GroupSeriesDev& S = ser[b];
  fit_z0_one(S.nz, S.zt, S.angles, S.sx, S.sy, S.sx64, S.sy64, S.rot, S.z0);
}

// max over err[order[i]] (the DoIt return value), initial -1e20, per series
__global__ void k_max_err_group(const GroupSeriesDev* __restrict__ ser,
                                const int* __restrict__ active, float* out) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0 || (active && active[b] == 0)) return;
  float m = -1e20f;
  for (int i = 0; i < ser[b].n; ++i) {
    float e = ser[b].err[ser[b].order[i]];
    if (e > m) m = e;
  }
  out[b] = m;
}

int fit_z0_group(Context* c, const GroupSeriesDev* ser, const int* active, int nseries,
                 cudaStream_t st) {
  k_fit_z0_group<<<nseries, 32, 0, st>>>(ser, active);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int max_err_group(Context* c, const GroupSeriesDev* ser, const int* active, int nseries,
                  float* d_out, cudaStream_t st) {
  k_max_err_group<<<nseries, 32, 0, st>>>(ser, active, d_out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

__device__ void fit_z0_one(int nz, int zt, const float* __restrict__ angles, float* sx,
                           float* sy, double* sx64, double* sy64, const float* __restrict__ rot,
                           float* z0p) {
  if (sx64 != nullptr) {
    double s0x, s0y;
    rot_shift64(sx64[zt], sy64[zt], -rot[zt], &s0x, &s0y);
    const double cent0 = s0x / cos((double)angles[zt] * kD2R);
    double dA = 0.0, dB = 0.0;
    for (int i = 0; i < nz; ++i) {
      double r0, r1;
      rot_shift64(sx64[i], sy64[i], -rot[i], &r0, &r1);
      const double ds = sin((double)angles[i] * kD2R), dc = cos((double)angles[i] * kD2R);
      dA += (cent0 * dc - r0) * ds;
      dB += ds * ds;
    }
    const float z0 = (float)(dA / (dB + 1e-30));
    *z0p = z0;
    if (z0 == 0.0f) return;
    for (int i = 0; i < nz; ++i) {
      if (i == zt) continue;
      double a, b;
      z_induced64(z0, angles[i], rot[i], &a, &b);
      sx64[i] -= a;
      sy64[i] -= b;
      sx[i] = (float)sx64[i];
      sy[i] = (float)sy64[i];
    }
    return;
  }
  float s0x, s0y;
  rot_shift(sx[zt], sy[zt], -rot[zt], &s0x, &s0y);
  float cent0 = (float)((double)s0x / cos((double)angles[zt] * kD2R));
  double dA = 0.0, dB = 0.0;
  for (int i = 0; i < nz; ++i) {
    float r0, r1;
    rot_shift(sx[i], sy[i], -rot[i], &r0, &r1);
    double ds = sin((double)angles[i] * kD2R), dc = cos((double)angles[i] * kD2R);
    dA += ((double)cent0 * dc - (double)r0) * ds;
    dB += ds * ds;
  }
  float z0 = (float)(dA / (dB + 1e-30));
  *z0p = z0;
  if (z0 == 0.0f) return;
  for (int i = 0; i < nz; ++i) {
    if (i == zt) continue;
    float a, b;
    z_induced(z0, angles[i], rot[i], &a, &b);
    sx[i] = __fadd_rn(sx[i], __fmul_rn(a, -1.0f));
    sy[i] = __fadd_rn(sy[i], __fmul_rn(b, -1.0f));
  }
}

int fit_z0(Context* c, int nz, int zt, const float* d_angles, float* d_sx, float* d_sy,
           double* d_sx64, double* d_sy64, const float* d_rot, float* d_z0, cudaStream_t st) {
  k_fit_z0<<<1, 32, 0, st>>>(nz, zt, d_angles, d_sx, d_sy, d_sx64, d_sy64, d_rot, d_z0);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// max over err[i] for i in list (the DoIt return value), initial -1e20.
__global__ void k_max_err(const float* __restrict__ err, const int* __restrict__ order, int n,
                          float* out) {
  if (threadIdx.x != 0) return;
  float m = -1e20f;
  for (int i = 0; i < n; ++i) {
    float e = err[order[i]];
    if (e > m) m = e;
  }
  *out = m;
}

int max_err(Context* c, const float* d_err, const int* d_order, int n, float* d_out,
            cudaStream_t st) {
  k_max_err<<<1, 32, 0, st>>>(d_err, d_order, n, d_out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Stretch about the tilt axis (CalcCC.cu:8-46, 149-171).  One map per z slice of
// the grid; matrices m[3*j..].  Rows of `stride` floats, `gw` columns computed.
__device__ __forceinline__ float stretch_random(float X, float Y, int width, int height,
                                                int grid_x, const float* in) {
  int x = (int)fabsf(X), y = (int)fabsf(Y);
  if (x >= width) x = width - 1 - (x % (width - 1));
  if (y >= height) y = height - 1 - (y % (height - 1));
  const int win = 31, size = win * win;
  unsigned int next = (unsigned int)(y * width + x);
  for (int i = 0; i < size; ++i) {
    next = (next * 7u) % (unsigned int)size;
    int ix = (int)(next % (unsigned int)size) - win / 2 + x;
    if (ix < 0 || ix >= width) continue;
    int iy = (int)(next / (unsigned int)win) - win / 2 + y;
    if (iy < 0 || iy >= height) continue;
    return in[iy * width + ix];
  }
  return in[height / 2 * width + grid_x / 2];
}

__device__ __forceinline__ float stretch_pixel(const float* in, int x, int y, int gw, int h,
                                               int stride, float m0, float m1, float m2,
                                               bool randfill) {
  float X = __fadd_rn(__fsub_rn((float)x, __fmul_rn(0.5f, (float)gw)), 0.5f);
  float Y = (float)((double)y - 0.5 * (double)h + 0.5);
  float buf = __fadd_rn(__fmul_rn(X, m0), __fmul_rn(Y, m1));
  Y = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(X, m1), __fmul_rn(Y, m2)), __fmul_rn(0.5f, (float)h)),
                0.5f);
  X = __fsub_rn(__fadd_rn(buf, __fmul_rn(0.5f, (float)gw)), 0.5f);
  if (X >= 0.0f && X < (float)(gw - 1) && Y >= 0.0f && Y < (float)(h - 1)) {
    int ix = (int)X, iy = (int)Y;
    int i = iy * stride + ix;
    float fx = __fsub_rn(X, (float)ix), fy = __fsub_rn(Y, (float)iy);
    float f2 = __fsub_rn(1.0f, fx), f3 = __fsub_rn(1.0f, fy);
    float v = __fmul_rn(__fmul_rn(in[i], f2), f3);
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + 1], fx), f3));
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + stride], f2), fy));
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + stride + 1], fx), fy));
    return v;
  }
  if (randfill) return stretch_random(X, Y, stride, h, gw, in);
  return kSentinel;
}

__global__ void k_stretch(const float* __restrict__ src, size_t src_img_stride,
                          const int* __restrict__ src_idx, int gw, int h, int stride,
                          const float* __restrict__ mats, int randfill, float* __restrict__ dst,
                          size_t dst_img_stride) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  int j = blockIdx.z;
  if (x >= gw || y >= h) return;
  const float* in = src + (size_t)src_idx[j] * src_img_stride;
  const float* m = mats + 3 * j;
  dst[(size_t)j * dst_img_stride + (size_t)y * stride + x] =
      stretch_pixel(in, x, y, gw, h, stride, m[0], m[1], m[2], randfill != 0);
}

int stretch_many(Context* c, const float* src, size_t src_img_stride, const int* d_src_idx,
                 int gw, int h, int stride, const float* d_mats, int n, int randfill, float* dst,
                 size_t dst_img_stride, cudaStream_t st) {
  dim3 blk(64, 4), grd((gw + 63) / 64, (h + 3) / 4, n);
  k_stretch<<<grd, blk, 0, st>>>(src, src_img_stride, d_src_idx, gw, h, stride, d_mats, randfill,
                                 dst, dst_img_stride);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// CalcCC::Stretch matrix (CalcCC.cu:318-332); the stretch factor arrives as float.
void stretch_matrix(float dstretch, float tilt_axis, float* m) {
  double d2t = 2 * kD2R * (double)tilt_axis;
  double s2 = std::sin(d2t), c2 = std::cos(d2t);
  double P = 0.5 * ((double)dstretch + 1), M = 0.5 * ((double)dstretch - 1);
  float a0 = (float)(P + M * c2), a1 = (float)(1 * M * s2), a2 = (float)(P - M * c2);
  float det = a0 * a2 - a1 * a1;
  m[0] = a2 / det;
  m[1] = -a1 / det;
  m[2] = a0 / det;
}

}  // namespace mf
