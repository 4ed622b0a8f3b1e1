// Common-line tilt-axis search (reference: Markerfree/src/method/Rotate.cu).
//
// The reference processes one tilt at a time: it reads the slice from disk,
// launches GRadon for the 100 candidate axes, then per line a mean kernel, a
// window kernel and a batch-1 cuFFT, copies the spectra to the host, and scores
// every candidate with per-tilt cudaMalloc/cudaFree and two device-to-host
// copies.  Here every tilt stays in HBM: one launch samples all (tilt,
// candidate, line position) Radon lines, one launch windows all lines, one
// batched cuFFT transforms them, and two launches score all candidates.
#include <cfloat>

#include "mf_xcorr.hpp"

namespace mf {

// GCalcCommonRegion (Rotate.cu:9-40); entries whose first step already leaves
// the image stay 0 here (the reference leaves them unset).
__global__ void k_common_region(int width, int height, int L, const float2* __restrict__ cs,
                                float shift_x, float shift_y, int* __restrict__ region) {
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (y >= L) return;
  int i = blockIdx.x * L + y;
  float fsin = cs[blockIdx.x].y, fcos = cs[blockIdx.x].x;
  int half = L / 2;
  float ox = __fadd_rn(__fmul_rn((float)width, 0.5f), shift_x);
  float oy = __fadd_rn(__fmul_rn((float)height, 0.5f), shift_y);
  float fy = __fsub_rn((float)y, __fmul_rn((float)L, 0.5f));
  int left = 0, right = 0;
  for (int x = 1; x < half; ++x) {
    float X = __fadd_rn(__fsub_rn(__fmul_rn((float)(-x), fcos), __fmul_rn(fy, fsin)), ox);
    float Y = __fadd_rn(__fadd_rn(__fmul_rn((float)(-x), fsin), __fmul_rn(fy, fcos)), oy);
    if (X < 0 || X >= width) break;
    if (Y < 0 || Y >= height) break;
    left = -x;
  }
  for (int x = 1; x < half; ++x) {
    float X = __fadd_rn(__fsub_rn(__fmul_rn((float)x, fcos), __fmul_rn(fy, fsin)), ox);
    float Y = __fadd_rn(__fadd_rn(__fmul_rn((float)x, fsin), __fmul_rn(fy, fcos)), oy);
    if (X < 0 || X >= width) break;
    if (Y < 0 || Y >= height) break;
    right = x;
  }
  region[2 * i] = left;
  region[2 * i + 1] = right;
}

// GRadon (Rotate.cu:42-95) for every tilt z = blockIdx.z.
__global__ void k_radon(const float* __restrict__ stack, int width, int height, int L, int num,
                        const float2* __restrict__ cs, const float* __restrict__ tilt_cos,
                        const float* __restrict__ sxs, const float* __restrict__ sys,
                        const int* __restrict__ region, float* __restrict__ lines) {
  int y = blockIdx.y * blockDim.x + threadIdx.x;
  int b = blockIdx.x;
  int z = blockIdx.z;
  if (y >= L) return;
  const float* proj = stack + (size_t)z * width * height;
  float fsr = cs[b].y, fcr = cs[b].x;
  float fy = __fsub_rn((float)y, __fmul_rn((float)L, 0.5f));
  float ox = __fadd_rn(__fmul_rn((float)width, 0.5f), sxs[z]);
  float oy = __fadd_rn(__fmul_rn((float)height, 0.5f), sys[z]);
  float fc = tilt_cos[z];
  int i = b * L + y;
  float sum = 0.0f;
  int cnt = 0;
  int left = (int)__fadd_rn(__fmul_rn((float)region[2 * i], fc), 0.5f);
  int right = (int)__fadd_rn(__fmul_rn((float)region[2 * i + 1], fc), 0.5f);
  // left <= 0 <= right, so one loop visits the reference's two loops in order;
  // fy*sin and fy*cos are loop invariant with the same rounding as the reference.
  // The float copy of x is stepped by 1.0 (exact below 2^24) instead of converted,
  // and the in-range coordinates (0 <= X < 2^23) are truncated by a round-toward-
  // zero add of 2^23, which gives the same integer as (int)X.
  const float ys = __fmul_rn(fy, fsr), yc = __fmul_rn(fy, fcr);
  const float fw = (float)width, fh = (float)height;
  float fx = (float)left;
  for (int x = left; x < right; ++x, fx = __fadd_rn(fx, 1.0f)) {
    float X = __fadd_rn(__fsub_rn(__fmul_rn(fx, fcr), ys), ox);
    float Y = __fadd_rn(__fadd_rn(__fmul_rn(fx, fsr), yc), oy);
    if (!(X >= 0.0f && X < fw && Y >= 0.0f && Y < fh)) continue;
    int ix = __float_as_int(__fadd_rz(X, 8388608.0f)) - 0x4B000000;
    int iy = __float_as_int(__fadd_rz(Y, 8388608.0f)) - 0x4B000000;
    float v = __ldg(proj + (size_t)iy * width + ix);
    if (v < 0) continue;
    sum = __fadd_rn(sum, v);
    cnt++;
  }
  lines[((size_t)z * num + b) * (L + 2) + y] = (cnt == 0) ? kSentinel : __fdiv_rn(sum, (float)cnt);
}

// GCalcMean + GRemoveMean (Rotate.cu:97-157) for one line per block.
__global__ void k_line_prep(float* __restrict__ lines, int L) {
  __shared__ double s_sum[256];
  __shared__ int s_cnt[256];
  float* p = lines + (size_t)blockIdx.x * (L + 2);
  double a = 0.0;
  int n = 0;
  for (int y = threadIdx.x; y < L; y += blockDim.x) {
    float v = p[y];
    if (v > -1e10f) {
      a += v;
      n++;
    }
  }
  s_sum[threadIdx.x] = a;
  s_cnt[threadIdx.x] = n;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + h];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + h];
    }
    __syncthreads();
  }
  float mean = s_cnt[0] == 0 ? 0.0f : (float)(s_sum[0] / s_cnt[0]);
  __syncthreads();
  float half = __fmul_rn(0.5f, (float)L);
  for (int y = threadIdx.x; y < L; y += blockDim.x) {
    float v = p[y];
    if (v < 0)
      v = 0.0f;
    else
      v = __fsub_rn(v, mean);
    float fr = __fdiv_rn(fabsf(__fsub_rn((float)y, half)), half);
    fr = __fmul_rn(0.5f, __fsub_rn(1.0f, (float)cos((double)(float)(3.14159 * (double)fr))));
    fr = __fsub_rn(1.0f, powf(fr, 100.0f));
    p[y] = __fmul_rn(v, __fmul_rn(fr, fr));
  }
}

// Sum of the candidate's spectra over tilts (GSumCmp with factors 1, 1).
__global__ void k_axis_sum(const cufftComplex* __restrict__ spec, int nz, int num, int cmp,
                           cufftComplex* __restrict__ sum) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y;
  if (k >= cmp) return;
  float re = 0.0f, im = 0.0f;
  for (int z = 0; z < nz; ++z) {
    cufftComplex v = spec[((size_t)z * num + b) * cmp + k];
    re = __fadd_rn(re, v.x);
    im = __fadd_rn(im, v.y);
  }
  sum[(size_t)b * cmp + k] = make_cuComplex(re, im);
}

// GConv (1-D, B = 10) + GSum (Rotate.cu:179-251) for (candidate b, tilt z).
__global__ void k_axis_cc(const cufftComplex* __restrict__ spec,
                          const cufftComplex* __restrict__ sum, int nz, int num, int cmp,
                          float* __restrict__ cc_out) {
  __shared__ double s_cc[128], s_sd[128];
  int b = blockIdx.x, z = blockIdx.y;
  const cufftComplex* line = spec + ((size_t)z * num + b) * cmp;
  const cufftComplex* sm = sum + (size_t)b * cmp;
  double cc = 0.0, sd = 0.0;
  for (int k = 1 + threadIdx.x; k < cmp; k += blockDim.x) {
    cufftComplex l = line[k], s = sm[k];
    float rr = __fsub_rn(s.x, l.x), ri = __fsub_rn(s.y, l.y);  // sum*1 + line*(-1)
    float f = __fdiv_rn((float)k, __fmul_rn(2.0f, (float)(cmp - 1)));
    f = (float)exp((double)__fmul_rn(__fmul_rn(-20.0f, f), f));
    float a1 = sqrtf(__fadd_rn(__fmul_rn(rr, rr), __fmul_rn(ri, ri)));
    float a2 = sqrtf(__fadd_rn(__fmul_rn(l.x, l.x), __fmul_rn(l.y, l.y)));
    float num_ = __fmul_rn(__fadd_rn(__fmul_rn(l.x, rr), __fmul_rn(l.y, ri)), f);
    cc += (double)__fdiv_rn(num_, __fadd_rn(__fmul_rn(a1, a2), 1e-20f));
    sd += (double)f;
  }
  s_cc[threadIdx.x] = cc;
  s_sd[threadIdx.x] = sd;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      s_cc[threadIdx.x] += s_cc[threadIdx.x + h];
      s_sd[threadIdx.x] += s_sd[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) cc_out[(size_t)b * nz + z] = __fdiv_rn((float)s_cc[0], (float)s_sd[0]);
}

__global__ void k_axis_score(const float* __restrict__ cc, int nz, int num,
                             float* __restrict__ score) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= num) return;
  float s = 0.0f;
  for (int z = 0; z < nz; ++z) s = __fadd_rn(s, cc[(size_t)b * nz + z]);
  score[b] = __fdiv_rn(s, (float)nz);
}

struct AxisBuffers {
  DevBuf cs, tcos, sx, sy, region, lines, sum, cc, score;
};

int tilt_axis_scores(Context* c, cufftHandle plan, const float* stack, int nx, int ny, int nz,
                     const float* angles,
                     const float* sx, const float* sy, int zt, const float* rot_cand, int num,
                     int L, std::vector<float>* scores, cudaStream_t st) {
  const int cmp = L / 2 + 1;
  AxisBuffers B;
  std::vector<float2> cs(num);
  for (int b = 0; b < num; ++b) {
    float a = rot_cand[b] * 3.1415926f / 180.0f;
    cs[b] = make_float2(cos_f(a), sin_f(a));
  }
  std::vector<float> tc(nz);
  for (int z = 0; z < nz; ++z) tc[z] = (float)std::cos(angles[z] * kD2R);
  MF_TRY(B.cs.alloc(sizeof(float2) * num));
  MF_TRY(B.tcos.alloc(sizeof(float) * nz));
  MF_TRY(B.sx.alloc(sizeof(float) * nz));
  MF_TRY(B.sy.alloc(sizeof(float) * nz));
  MF_TRY(B.region.alloc(sizeof(int) * 2 * (size_t)num * L));
  MF_TRY(B.lines.alloc(sizeof(float) * (size_t)nz * num * (L + 2)));
  MF_TRY(B.sum.alloc(sizeof(cufftComplex) * (size_t)num * cmp));
  MF_TRY(B.cc.alloc(sizeof(float) * (size_t)num * nz));
  MF_TRY(B.score.alloc(sizeof(float) * num));
  MF_CHECK_CUDA(cudaMemcpyAsync(B.cs.p, cs.data(), sizeof(float2) * num, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(B.tcos.p, tc.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(B.sx.p, sx, sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(B.sy.p, sy, sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  k_common_region<<<dim3(num, (L + 127) / 128), dim3(1, 128), 0, st>>>(
      nx, ny, L, B.cs.as<float2>(), sx[zt], sy[zt], B.region.as<int>());
  k_radon<<<dim3(num, (L + 127) / 128, nz), 128, 0, st>>>(
      stack, nx, ny, L, num, B.cs.as<float2>(), B.tcos.as<float>(), B.sx.as<float>(),
      B.sy.as<float>(), B.region.as<int>(), B.lines.as<float>());
  k_line_prep<<<nz * num, 256, 0, st>>>(B.lines.as<float>(), L);
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  MF_CHECK_CUFFT(cufftExecR2C(plan, B.lines.as<cufftReal>(), B.lines.as<cufftComplex>()));
  const cufftComplex* spec = B.lines.as<cufftComplex>();
  k_axis_sum<<<dim3((cmp + 127) / 128, num), 128, 0, st>>>(spec, nz, num, cmp,
                                                            B.sum.as<cufftComplex>());
  k_axis_cc<<<dim3(num, nz), 128, 0, st>>>(spec, B.sum.as<cufftComplex>(), nz, num, cmp,
                                           B.cc.as<float>());
  k_axis_score<<<(num + 127) / 128, 128, 0, st>>>(B.cc.as<float>(), nz, num, B.score.as<float>());
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  scores->resize(num);
  MF_CHECK_CUDA(cudaMemcpyAsync(scores->data(), B.score.p, sizeof(float) * num,
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// ---------------------------------------------------------------------------
// FindOffset::Correlate moments (FindOffset.cu:7-72, 176-238) for many
// (offset, tilt pair) entries at once; the stretched image is evaluated on the fly.
__device__ __forceinline__ float stretch_nofill(const float* in, int x, int y, int w, int h,
                                                float m0, float m1, float m2) {
  float X = __fadd_rn(__fsub_rn((float)x, __fmul_rn(0.5f, (float)w)), 0.5f);
  float Y = (float)((double)y - 0.5 * (double)h + 0.5);
  float buf = __fadd_rn(__fmul_rn(X, m0), __fmul_rn(Y, m1));
  Y = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(X, m1), __fmul_rn(Y, m2)), __fmul_rn(0.5f, (float)h)),
                0.5f);
  X = __fsub_rn(__fadd_rn(buf, __fmul_rn(0.5f, (float)w)), 0.5f);
  if (X >= 0.0f && X < (float)(w - 1) && Y >= 0.0f && Y < (float)(h - 1)) {
    int ix = (int)X, iy = (int)Y;
    int i = iy * w + ix;
    float fx = __fsub_rn(X, (float)ix), fy = __fsub_rn(Y, (float)iy);
    float f2 = __fsub_rn(1.0f, fx), f3 = __fsub_rn(1.0f, fy);
    float v = __fmul_rn(__fmul_rn(in[i], f2), f3);
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + 1], fx), f3));
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + w], f2), fy));
    v = __fadd_rn(v, __fmul_rn(__fmul_rn(in[i + w + 1], fx), fy));
    return v;
  }
  return kSentinel;
}

__global__ void k_offset_moments(const float* __restrict__ corr, int w, int h,
                                 const OffsetPair* __restrict__ pairs, double* __restrict__ out) {
  __shared__ double s[6][256];
  OffsetPair p = pairs[blockIdx.x];
  const float* ref = corr + (size_t)p.ref * w * h;
  const float* img = corr + (size_t)p.img * w * h;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
    int y = i / w, x = i % w;
    float v1 = ref[i];
    if (v1 < -1e10f) continue;
    float v2 = stretch_nofill(img, x, y, w, h, p.m0, p.m1, p.m2);
    if (v2 < -1e10f) continue;
    a[0] += v1;
    a[1] += v2;
    a[2] += (double)__fmul_rn(v1, v1);
    a[3] += (double)__fmul_rn(v2, v2);
    a[4] += (double)__fmul_rn(v1, v2);
    a[5] += 1.0;
  }
  for (int k = 0; k < 6; ++k) s[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
    if (threadIdx.x < hh)
      for (int k = 0; k < 6; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + hh];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) out[(size_t)blockIdx.x * 6 + k] = s[k][0];
}

int offset_moments(Context* c, const float* corr, int w, int h, const OffsetPair* d_pairs,
                   int npairs, double* d_out, cudaStream_t st) {
  k_offset_moments<<<npairs, 256, 0, st>>>(corr, w, h, d_pairs, d_out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

}  // namespace mf
