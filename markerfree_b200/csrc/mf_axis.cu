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

// Arithmetic of the reference's device code.  nvcc contracts a*b + c into one
// fused multiply-add (its default), taking the first product of a sum of two
// products as the fused one: x*c - y*s + o becomes fma(x, c, -(y*s)) + o.  The
// candidate angles' sine and cosine are CUDA's sinf/cosf of the same float
// argument, as in the reference.  Emulating both keeps the sampled pixels and
// the line values those of the reference binary.
__device__ __forceinline__ float lin2(float x, float c, float yprod, float o) {
  return __fadd_rn(__fmaf_rn(x, c, yprod), o);
}

// CUDA's cosf and sinf of each argument, as the kernels evaluate them.
__global__ void k_cos_sin(const float* __restrict__ x, int n, float* __restrict__ c,
                          float* __restrict__ s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  c[i] = cosf(x[i]);
  s[i] = sinf(x[i]);
}

int device_cos_sin(Context* ctx, const float* d_x, int n, float* d_c, float* d_s,
                   cudaStream_t st) {
  if (n <= 0) return MF_OK;
  k_cos_sin<<<(n + 255) / 256, 256, 0, st>>>(d_x, n, d_c, d_s);
  ctx->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// cs[b] = (cosf(a), sinf(a)), a = rot[b] * 3.1415926f / 180.0f (Rotate.cu:16-18, 50-52)
__global__ void k_axis_cs(const float* __restrict__ rot, int num, float2* __restrict__ cs) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= num) return;
  const float a = __fdiv_rn(__fmul_rn(rot[b], 3.1415926f), 180.0f);
  cs[b] = make_float2(cosf(a), sinf(a));
}

// Smallest x in [a, b) with pred(x), for a predicate that is false then true
// along x; b when it is never true.
template <class P>
__device__ __forceinline__ int first_true(int a, int b, P pred) {
  while (a < b) {
    const int m = a + ((b - a) >> 1);
    if (pred(m))
      b = m;
    else
      a = m + 1;
  }
  return a;
}

// GCalcCommonRegion (Rotate.cu:9-40); entries whose first step already leaves
// the image stay 0 here (the reference leaves them unset).
__global__ void k_common_region(int width, int height, int L, const float2* __restrict__ cs,
                                float shift_x, float shift_y, int* __restrict__ region) {
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (y >= L) return;
  int i = blockIdx.x * L + y;
  float fsin = cs[blockIdx.x].y, fcos = cs[blockIdx.x].x;
  int half = L / 2;
  float ox = __fmaf_rn((float)width, 0.5f, shift_x);
  float oy = __fmaf_rn((float)height, 0.5f, shift_y);
  float fy = __fmaf_rn(-(float)L, 0.5f, (float)y);
  const float ys = -__fmul_rn(fy, fsin), yc = __fmul_rn(fy, fcos);
  // The reference walks outwards from the centre and stops at the first sample
  // outside the image.  The sample coordinates are monotone in x (every step is a
  // correctly rounded monotone operation), so the samples inside the image form
  // one interval of x and the first one outside on each side is found by
  // bisection: the same ends as the walk.
  const float fw = (float)width, fh = (float)height;
  auto inside = [&](int x) {
    const float X = lin2((float)x, fcos, ys, ox), Y = lin2((float)x, fsin, yc, oy);
    return !(X < 0 || X >= fw) && !(Y < 0 || Y >= fh);
  };
  int left = 0, right = 0;
  if (half > 1 && inside(-1)) left = -(first_true(2, half, [&](int x) { return !inside(-x); }) - 1);
  if (half > 1 && inside(1)) right = first_true(2, half, [&](int x) { return !inside(x); }) - 1;
  region[2 * i] = left;
  region[2 * i + 1] = right;
}

// Sample coordinates of GRadon (Rotate.cu:62-63, 76-77): X = x cos - y sin + ox,
// Y = x sin + y cos + oy, contracted as the reference's device code is.
struct RadonLine {
  float c, s, ys, yc, ox, oy;  // ys = -(y sin), yc = y cos
  __device__ __forceinline__ float X(float fx) const { return lin2(fx, c, ys, ox); }
  __device__ __forceinline__ float Y(float fx) const { return lin2(fx, s, yc, oy); }
};

// Sub-interval of [a, b) on which 0 <= f(x) < lim, for f = rounded (x k + consts):
// f is monotone in x (non-decreasing for k >= 0, non-increasing for k < 0) because
// every step (the fused x k + c, then + o) is a correctly rounded monotone
// operation, so the set is an interval.
template <class F>
__device__ __forceinline__ void in_range(int* a, int* b, float k, float lim, F f) {
  if (*a >= *b) return;
  if (k >= 0.0f) {
    *a = first_true(*a, *b, [&](int x) { return f((float)x) >= 0.0f; });
    *b = first_true(*a, *b, [&](int x) { return !(f((float)x) < lim); });
  } else {
    *a = first_true(*a, *b, [&](int x) { return f((float)x) < lim; });
    *b = first_true(*a, *b, [&](int x) { return !(f((float)x) >= 0.0f); });
  }
}

// Column-major copy of every tilt image: out[z][x][y] = in[z][y][x]; neg[z] is set
// to 1 when image z holds a value below zero (the caller zeroes neg first).
__global__ void k_transpose_stack(const float* __restrict__ in, int width, int height,
                                  float* __restrict__ out, int* __restrict__ neg) {
  __shared__ float tile[32][33];
  const size_t pix = (size_t)width * height;
  const float* src = in + blockIdx.z * pix;
  float* dst = out + blockIdx.z * pix;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  bool below = false;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int x = x0 + threadIdx.x, y = y0 + j;
    if (x < width && y < height) {
      const float v = src[(size_t)y * width + x];
      below = below || v < 0.0f;
      tile[j][threadIdx.x] = v;
    }
  }
  if (below) neg[blockIdx.z] = 1;
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int y = y0 + threadIdx.x, x = x0 + j;
    if (x < width && y < height) dst[(size_t)x * height + y] = tile[threadIdx.x][j];
  }
}

int transpose_stack(Context* c, const float* stack, int width, int height, int nz, float* out,
                    int* neg, cudaStream_t st) {
  MF_CHECK_CUDA(cudaMemsetAsync(neg, 0, sizeof(int) * nz, st));
  k_transpose_stack<<<dim3((width + 31) / 32, (height + 31) / 32, nz), dim3(32, 8), 0, st>>>(
      stack, width, height, out, neg);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Two floats in one 64-bit register, for the packed f32x2 arithmetic of sm_100:
// each lane of fma.rn.f32x2 / add.rn.f32x2 / add.rz.f32x2 is the scalar IEEE
// operation with that rounding, so (X, Y) come out bit for bit as from
// __fmaf_rn / __fadd_rn / __fadd_rz, with one instruction for both coordinates.
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float* a, float* b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(*a), "=f"(*b) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma2_rn(unsigned long long a, unsigned long long b,
                                                      unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ unsigned long long add2_rn(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long add2_rz(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// Sum and count of the samples x in [lo, hi) of one line, every one of which is
// inside the image.  kByColumn: pixel (ix, iy) is proj[ix * stride + iy] (the
// column-major copy, stride = height), else proj[iy * stride + ix] (stride = width).
// kNonNeg: the image holds no value below zero, so the reference's skip of such
// samples never fires and every sample counts.
// An in-range coordinate (0 <= X < 2^23) is truncated by a round-toward-zero add
// of 2^23: the low bits of the sum are (int)X, and the index is formed from the
// biased bits in 32-bit modular arithmetic.  kFold (stride a multiple of 256):
// 2^23's bits times the stride vanish mod 2^32, so the biased index is the true
// index plus 0x4B000000 without wrapping, and that constant moves into the base
// address instead of being subtracted per sample.
// Two consecutive samples are stepped together: each packed f32x2 operation
// evaluates one coordinate of samples x and x + 1 (lane for lane the scalar IEEE
// operation), and the samples are added to the sum in order, x first.
#ifndef MF_RADON_UNROLL
#define MF_RADON_UNROLL 4
#endif
#define MF_RADON_PRAGMA_(x) _Pragma(#x)
#define MF_RADON_PRAGMA(x) MF_RADON_PRAGMA_(x)
#define MF_RADON_UNROLL_PRAGMA MF_RADON_PRAGMA(unroll MF_RADON_UNROLL)
// kSh > 0 (stride = 2^kSh): the byte offset is formed by shifts alone,
// (slow bits << (kSh + 2)) + (fast bits << 2) in 32-bit arithmetic: the slow
// coordinate's bias vanishes (2^23 << (kSh + 2) is a multiple of 2^32), the fast
// one's leaves 4 * 2^23 mod 2^32 = 0x2C000000, which moves into the base address.
// Shifts and adds run on the integer pipe, the multiply-add of the index on the
// FP32 pipe that the coordinates already fill.  (No wrap: 4 * index + 0x2C000000
// stays below 2^32 for images below 8.8e8 pixels.)
#ifndef MF_RADON_SHIFT
#define MF_RADON_SHIFT 1
#endif
template <bool kByColumn, bool kNonNeg, bool kFold, int kSh = 0>
__device__ __forceinline__ void radon_samples(const float* __restrict__ proj, int stride,
                                              const RadonLine& ln, int lo, int hi, float* sum_out,
                                              int* cnt_out) {
  constexpr unsigned kBias = 0x4B000000u;  // bits of 2^23
  const unsigned bias_idx = kFold ? 0u : kBias * (unsigned)stride + kBias;  // mod 2^32
  const uintptr_t base = kSh > 0 ? (uintptr_t)proj - 0x2C000000ull
                                 : (uintptr_t)proj - (kFold ? 4ull * kBias : 0ull);
  const unsigned long long c2 = pack2(ln.c, ln.c), s2 = pack2(ln.s, ln.s);
  const unsigned long long ys2 = pack2(ln.ys, ln.ys), yc2 = pack2(ln.yc, ln.yc);
  const unsigned long long ox2 = pack2(ln.ox, ln.ox), oy2 = pack2(ln.oy, ln.oy);
  const unsigned long long big2 = pack2(8388608.0f, 8388608.0f), two2 = pack2(2.0f, 2.0f);
  auto index = [&](float tx, float ty) -> unsigned {
    const unsigned bx = __float_as_uint(tx), by = __float_as_uint(ty);
    if (kSh > 0) {  // byte offset (see above)
      const unsigned slow = kByColumn ? bx : by, fast = kByColumn ? by : bx;
      return (slow << (kSh + 2)) + (fast << 2);
    }
    return (kByColumn ? bx * (unsigned)stride + by : by * (unsigned)stride + bx) - bias_idx;
  };
  auto load = [&](unsigned idx) -> float {
    if (kSh > 0) return __ldg(reinterpret_cast<const float*>(base + (uintptr_t)idx));
    return __ldg(reinterpret_cast<const float*>(base + ((uintptr_t)idx << 2)));
  };
  unsigned long long fx2 = pack2((float)lo, (float)(lo + 1));
  float sum = 0.0f;
  int cnt = 0;
  int x = lo;
  MF_RADON_UNROLL_PRAGMA
  for (; x + 1 < hi; x += 2) {
    // X = fma(x, cos, -(y sin)) + ox, Y = fma(x, sin, y cos) + oy, as lin2(), for x, x + 1
    const unsigned long long tx = add2_rz(add2_rn(fma2_rn(fx2, c2, ys2), ox2), big2);
    const unsigned long long ty = add2_rz(add2_rn(fma2_rn(fx2, s2, yc2), oy2), big2);
    fx2 = add2_rn(fx2, two2);
    float x0, x1, y0, y1;
    unpack2(tx, &x0, &x1);
    unpack2(ty, &y0, &y1);
    const float v0 = load(index(x0, y0));
    const float v1 = load(index(x1, y1));
    if (kNonNeg) {
      sum = __fadd_rn(sum, v0);
      sum = __fadd_rn(sum, v1);
    } else {
      if (!(v0 < 0)) {
        cnt++;
        sum = __fadd_rn(sum, v0);
      }
      if (!(v1 < 0)) {
        cnt++;
        sum = __fadd_rn(sum, v1);
      }
    }
  }
  if (x < hi) {
    const float fx = (float)x;
    const float tx = __fadd_rz(ln.X(fx), 8388608.0f), ty = __fadd_rz(ln.Y(fx), 8388608.0f);
    const float v = load(index(tx, ty));
    if (kNonNeg || !(v < 0)) {
      cnt++;
      sum = __fadd_rn(sum, v);
    }
  }
  *sum_out = sum;
  *cnt_out = kNonNeg ? max(hi - lo, 0) : cnt;
}

template <bool kByColumn, bool kNonNeg>
__device__ __forceinline__ void radon_line(const float* __restrict__ proj, int stride,
                                           const RadonLine& ln, int lo, int hi, float* sum,
                                           int* cnt) {
  if (MF_RADON_SHIFT && stride == 2048)
    radon_samples<kByColumn, kNonNeg, true, 11>(proj, stride, ln, lo, hi, sum, cnt);
  else if (MF_RADON_SHIFT && stride == 1024)
    radon_samples<kByColumn, kNonNeg, true, 10>(proj, stride, ln, lo, hi, sum, cnt);
  else if (MF_RADON_SHIFT && stride == 4096)
    radon_samples<kByColumn, kNonNeg, true, 12>(proj, stride, ln, lo, hi, sum, cnt);
  else if ((stride & 255) == 0)
    radon_samples<kByColumn, kNonNeg, true>(proj, stride, ln, lo, hi, sum, cnt);
  else
    radon_samples<kByColumn, kNonNeg, false>(proj, stride, ln, lo, hi, sum, cnt);
}

// GRadon (Rotate.cu:42-95) for every tilt z = blockIdx.z.  The samples that fall
// inside the image form one interval of x (the coordinates are monotone in x), so
// it is found once per line by bisection on the same rounded expressions and the
// loop then runs without bounds tests; the samples taken and their order (left
// to right, as the reference's two loops) are unchanged.
//
// Neighbouring lanes take neighbouring lines, whose samples at one x lie one
// step of (-sin, cos) apart.  For a steep candidate (|sin| >= |cos|) that step
// runs along an image row, so a warp reads one row segment from the row-major
// stack; otherwise it runs along a column and the warp reads the column-major copy
// `stack_t` instead.  Both hold the same values: only the address changes.
// The warps of a block take the same 32 lines of kRadonCand neighbouring
// candidates: their lines differ by a fraction of a degree, so at each x they
// gather from nearly the same pixels, and the block's warps share those cache
// lines in L1 instead of each fetching them from L2.
#ifndef MF_RADON_CAND
#define MF_RADON_CAND 4
#endif
constexpr int kRadonCand = MF_RADON_CAND;  // candidates (warps) per block

__global__ void __launch_bounds__(32 * kRadonCand)
    k_radon(const float* __restrict__ stack, const float* __restrict__ stack_t,
            const int* __restrict__ neg, int width, int height, int L, int num,
            const float2* __restrict__ cs, const float* __restrict__ tilt_cos,
            const float* __restrict__ sxs, const float* __restrict__ sys,
            const int* __restrict__ region, float* __restrict__ lines,
            unsigned long long* __restrict__ samples) {
  const int y = blockIdx.y * 32 + (threadIdx.x & 31);
  const int b = blockIdx.x * kRadonCand + (threadIdx.x >> 5);
  const int z = blockIdx.z;
  if (y >= L || b >= num) return;
  RadonLine ln;
  ln.s = cs[b].y;
  ln.c = cs[b].x;
  const float fy = __fmaf_rn(-(float)L, 0.5f, (float)y);
  ln.ox = __fmaf_rn((float)width, 0.5f, sxs[z]);
  ln.oy = __fmaf_rn((float)height, 0.5f, sys[z]);
  ln.ys = -__fmul_rn(fy, ln.s);
  ln.yc = __fmul_rn(fy, ln.c);
  const float fc = tilt_cos[z];
  const int i = b * L + y;
  // left <= 0 <= right, so one loop visits the reference's two loops in order
  int lo = (int)__fmaf_rn((float)region[2 * i], fc, 0.5f);
  int hi = (int)__fmaf_rn((float)region[2 * i + 1], fc, 0.5f);
  const float fw = (float)width, fh = (float)height;
  in_range(&lo, &hi, ln.c, fw, [&](float fx) { return ln.X(fx); });
  in_range(&lo, &hi, ln.s, fh, [&](float fx) { return ln.Y(fx); });
  const size_t off = (size_t)z * width * height;
  float sum;
  int cnt;
  const bool nonneg = neg != nullptr && neg[z] == 0;
  if (stack_t != nullptr && fabsf(ln.c) > fabsf(ln.s)) {  // uniform over the warp
    if (nonneg)
      radon_line<true, true>(stack_t + off, height, ln, lo, hi, &sum, &cnt);
    else
      radon_line<true, false>(stack_t + off, height, ln, lo, hi, &sum, &cnt);
  } else {
    if (nonneg)
      radon_line<false, true>(stack + off, width, ln, lo, hi, &sum, &cnt);
    else
      radon_line<false, false>(stack + off, width, ln, lo, hi, &sum, &cnt);
  }
  lines[((size_t)z * num + b) * (L + 2) + y] = (cnt == 0) ? kSentinel : __fdiv_rn(sum, (float)cnt);
  if (samples) {  // stage timing: samples taken (one atomic per warp)
    const unsigned m = __activemask();
    const unsigned n = __reduce_add_sync(m, (unsigned)max(hi - lo, 0));
    if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(samples, (unsigned long long)n);
  }
}

// GCalcMean + GRemoveMean (Rotate.cu:97-157) for one line per block of 512
// threads: float partial sums over x = tid, tid + 512, ..., then the same
// shared-memory tree; the window's cosine is CUDA's cosf of the same argument.
__global__ void __launch_bounds__(512) k_line_prep(float* __restrict__ lines, int L) {
  __shared__ float s_sum[512];
  __shared__ int s_cnt[512];
  float* p = lines + (size_t)blockIdx.x * (L + 2);
  float a = 0.0f;
  int n = 0;
  for (int y = threadIdx.x; y < L; y += blockDim.x) {
    float v = p[y];
    if (v > -1e10f) {
      a = __fadd_rn(a, v);
      n++;
    }
  }
  s_sum[threadIdx.x] = a;
  s_cnt[threadIdx.x] = n;
  __syncthreads();
  for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      s_sum[threadIdx.x] = __fadd_rn(s_sum[threadIdx.x], s_sum[threadIdx.x + h]);
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + h];
    }
    __syncthreads();
  }
  const float mean = s_cnt[0] == 0 ? 0.0f : __fdiv_rn(s_sum[0], (float)s_cnt[0]);
  __syncthreads();
  const float half = __fmul_rn(0.5f, (float)L);
  for (int y = threadIdx.x; y < L; y += blockDim.x) {
    float v = p[y];
    if (v < 0)
      v = 0.0f;
    else
      v = __fsub_rn(v, mean);
    float fr = __fdiv_rn(fabsf(__fsub_rn((float)y, half)), half);
    fr = __fmul_rn(0.5f, __fsub_rn(1.0f, cosf((float)(3.14159 * (double)fr))));
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

// GConv (1-D, B = 10) + GSum (Rotate.cu:179-251) for (candidate b, tilt z), with
// the reference's partition: GConv blocks of blockDim (= CalcWarps(cmp) * 32)
// threads, one element per thread, a float tree per block; then GSum over the
// block partials with gsum_threads threads (strided float sums, then a tree).
__global__ void __launch_bounds__(512) k_axis_cc(const cufftComplex* __restrict__ spec,
                                                 const cufftComplex* __restrict__ sum, int nz,
                                                 int num, int cmp, int gsum_threads,
                                                 float* __restrict__ cc_out) {
  __shared__ float s_cc[512], s_sd[512];
  __shared__ float p_cc[64], p_sd[64];
  const int b = blockIdx.x, z = blockIdx.y;
  const cufftComplex* line = spec + ((size_t)z * num + b) * cmp;
  const cufftComplex* sm = sum + (size_t)b * cmp;
  const int bs = blockDim.x, tid = threadIdx.x;
  const int nblk = cmp / bs + 1;
  for (int vb = 0; vb < nblk; ++vb) {
    const int i = vb * bs + tid;
    float cc = 0.0f, sd = 0.0f;
    if (i < cmp && i != 0) {
      const cufftComplex l = line[i], s = sm[i];
      const float rx = __fsub_rn(s.x, l.x), ry = __fsub_rn(s.y, l.y);  // sum*1 + line*(-1)
      float f = __fdiv_rn((float)i, __fmul_rn(2.0f, (float)(cmp - 1)));
      f = expf(__fmul_rn(__fmul_rn(-20.0f, f), f));
      const float a1 = sqrtf(__fmaf_rn(rx, rx, __fmul_rn(ry, ry)));
      const float a2 = sqrtf(__fmaf_rn(l.x, l.x, __fmul_rn(l.y, l.y)));
      const float dot = __fmaf_rn(l.x, rx, __fmul_rn(l.y, ry));
      cc = __fdiv_rn(__fmul_rn(dot, f), __fmaf_rn(a1, a2, 1e-20f));
      sd = f;
    }
    s_cc[tid] = cc;
    s_sd[tid] = sd;
    __syncthreads();
    for (int h = bs >> 1; h > 0; h >>= 1) {
      if (tid < h) {
        s_cc[tid] = __fadd_rn(s_cc[tid], s_cc[tid + h]);
        s_sd[tid] = __fadd_rn(s_sd[tid], s_sd[tid + h]);
      }
      __syncthreads();
    }
    if (tid == 0) {
      p_cc[vb] = s_cc[0];
      p_sd[vb] = s_sd[0];
    }
    __syncthreads();
  }
  // GSum over the nblk partials
  float cc = 0.0f, sd = 0.0f;
  if (tid < gsum_threads)
    for (int x = tid; x < nblk; x += gsum_threads) {
      cc = __fadd_rn(cc, p_cc[x]);
      sd = __fadd_rn(sd, p_sd[x]);
    }
  s_cc[tid] = cc;
  s_sd[tid] = sd;
  __syncthreads();
  for (int h = gsum_threads >> 1; h > 0; h >>= 1) {
    if (tid < h) {
      s_cc[tid] = __fadd_rn(s_cc[tid], s_cc[tid + h]);
      s_sd[tid] = __fadd_rn(s_sd[tid], s_sd[tid + h]);
    }
    __syncthreads();
  }
  if (tid == 0) cc_out[(size_t)b * nz + z] = __fdiv_rn(s_cc[0], s_sd[0]);
}

// CalcTIltAxis::CalcWarps (Rotate.cu:563-572), host arithmetic as in the reference.
static int calc_warps(int size, int warp) {
  float fw = size / (float)warp;
  if (fw < 1.5f) return 1;
  int e = (int)(logf(fw) / logf(2.0f) + 0.5f);
  int w = 1 << e;
  return w > 16 ? 16 : w;
}

__global__ void k_axis_score(const float* __restrict__ cc, int nz, int num,
                             float* __restrict__ score) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= num) return;
  float s = 0.0f;
  for (int z = 0; z < nz; ++z) s = __fadd_rn(s, cc[(size_t)b * nz + z]);
  score[b] = __fdiv_rn(s, (float)nz);
}

AxisJob::~AxisJob() {
  if (ev[0]) cudaEventDestroy(ev[0]);
  if (ev[1]) cudaEventDestroy(ev[1]);
}

int tilt_axis_scores_enqueue(Context* c, cufftHandle plan, const float* stack,
                             const float* stack_t, const int* d_neg, int nx, int ny, int nz,
                             const float* angles, const float* sx, const float* sy, int zt,
                             const float* rot_cand, int num, int L, int slot, AxisJob* J,
                             cudaStream_t st) {
  const int cmp = L / 2 + 1;
  const int bs = calc_warps(cmp, 32) * 32;
  const int nblk = cmp / bs + 1;
  if (nblk > 64) return set_error(MF_ERR_ARG, "tilt axis: line of %d bins too long", L);
  const int gs = calc_warps(nblk, 32) * 32;
  J->num = num;
  J->L = L;
  J->nx = nx;
  J->ny = ny;
  J->nz = nz;
  char* host = (char*)c->pinned.get(slot, sizeof(float) * num + sizeof(unsigned long long));
  if (!host) return MF_ERR_NOMEM;
  J->h_count = (unsigned long long*)host;
  J->h_scores = (float*)(host + sizeof(unsigned long long));
  // device buffers are released stream-ordered when this function returns, after
  // the work queued here; only the page-locked results outlive it
  DevBuf rot, cs, tcos, d_sx, d_sy, region, lines, sum, cc, score, count;
  std::vector<float> tc(nz);
  for (int z = 0; z < nz; ++z) tc[z] = (float)std::cos(angles[z] * kD2R);
  MF_TRY(cs.alloc(sizeof(float2) * num));
  MF_TRY(tcos.alloc(sizeof(float) * nz));
  MF_TRY(d_sx.alloc(sizeof(float) * nz));
  MF_TRY(d_sy.alloc(sizeof(float) * nz));
  MF_TRY(region.alloc(sizeof(int) * 2 * (size_t)num * L));
  MF_TRY(lines.alloc(sizeof(float) * (size_t)nz * num * (L + 2)));
  MF_TRY(sum.alloc(sizeof(cufftComplex) * (size_t)num * cmp));
  MF_TRY(cc.alloc(sizeof(float) * (size_t)num * nz));
  MF_TRY(score.alloc(sizeof(float) * num));
  MF_TRY(rot.alloc(sizeof(float) * num));
  MF_CHECK_CUDA(cudaMemcpyAsync(rot.p, rot_cand, sizeof(float) * num, cudaMemcpyHostToDevice, st));
  k_axis_cs<<<(num + 127) / 128, 128, 0, st>>>(rot.as<float>(), num, cs.as<float2>());
  c->launches++;
  MF_CHECK_CUDA(cudaMemcpyAsync(tcos.p, tc.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_sx.p, sx, sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_sy.p, sy, sizeof(float) * nz, cudaMemcpyHostToDevice, st));
  k_common_region<<<dim3(num, (L + 127) / 128), dim3(1, 128), 0, st>>>(
      nx, ny, L, cs.as<float2>(), sx[zt], sy[zt], region.as<int>());
  // with stage timing on, the Radon kernel is timed on its own and counts its samples
  if (c->profiling) {
    MF_TRY(count.alloc(sizeof(unsigned long long)));
    MF_CHECK_CUDA(cudaMemsetAsync(count.p, 0, sizeof(unsigned long long), st));
    MF_CHECK_CUDA(cudaEventCreate(&J->ev[0]));
    MF_CHECK_CUDA(cudaEventCreate(&J->ev[1]));
    MF_CHECK_CUDA(cudaEventRecord(J->ev[0], st));
  }
  const dim3 rgrid((num + kRadonCand - 1) / kRadonCand, (L + 31) / 32, nz);
  k_radon<<<rgrid, 32 * kRadonCand, 0, st>>>(
      stack, stack_t, d_neg, nx, ny, L, num, cs.as<float2>(), tcos.as<float>(),
      d_sx.as<float>(), d_sy.as<float>(), region.as<int>(), lines.as<float>(),
      count.as<unsigned long long>());
  if (c->profiling) {
    MF_CHECK_CUDA(cudaEventRecord(J->ev[1], st));
    MF_CHECK_CUDA(cudaMemcpyAsync(J->h_count, count.p, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, st));
  }
  k_line_prep<<<nz * num, 512, 0, st>>>(lines.as<float>(), L);
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  MF_CHECK_CUFFT(cufftExecR2C(plan, lines.as<cufftReal>(), lines.as<cufftComplex>()));
  const cufftComplex* spec = lines.as<cufftComplex>();
  k_axis_sum<<<dim3((cmp + 127) / 128, num), 128, 0, st>>>(spec, nz, num, cmp,
                                                            sum.as<cufftComplex>());
  k_axis_cc<<<dim3(num, nz), bs, 0, st>>>(spec, sum.as<cufftComplex>(), nz, num, cmp, gs,
                                          cc.as<float>());
  k_axis_score<<<(num + 127) / 128, 128, 0, st>>>(cc.as<float>(), nz, num, score.as<float>());
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  MF_CHECK_CUDA(cudaMemcpyAsync(J->h_scores, score.p, sizeof(float) * num,
                                cudaMemcpyDeviceToHost, st));
  return MF_OK;
}

int tilt_axis_scores_finish(Context* c, AxisJob* J, std::vector<float>* scores) {
  if (J->ev[0]) {
    float ms = 0.0f;
    MF_CHECK_CUDA(cudaEventElapsedTime(&ms, J->ev[0], J->ev[1]));
    c->breakdown[kStageRadonMs] += ms;
    c->breakdown[kStageRadonSamples] += (double)*J->h_count;
    c->breakdown[kStageRadonLaunches] += 1.0;
    // compulsory bytes: every tilt image once, the line values written once
    c->breakdown[kStageRadonBytes] +=
        4.0 * (double)J->nx * J->ny * J->nz + 4.0 * (double)J->nz * J->num * (J->L + 2);
  }
  scores->assign(J->h_scores, J->h_scores + J->num);
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

// Each pair's image is split into kOffsetParts bands of rows, one block each; a
// block accumulates its band in FP64 and the bands are added in order.
constexpr int kOffsetParts = 16;

__global__ void k_offset_moments(const float* __restrict__ corr, int w, int h,
                                 const OffsetPair* __restrict__ pairs, double* __restrict__ part) {
  __shared__ double s[6][256];
  OffsetPair p = pairs[blockIdx.x];
  const float* ref = corr + (size_t)p.ref * w * h;
  const float* img = corr + (size_t)p.img * w * h;
  const int y0 = h * (int)blockIdx.y / kOffsetParts, y1 = h * ((int)blockIdx.y + 1) / kOffsetParts;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int y = y0; y < y1; ++y)
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
      float v1 = ref[(size_t)y * w + x];
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
    for (int k = 0; k < 6; ++k)
      part[((size_t)blockIdx.x * kOffsetParts + blockIdx.y) * 6 + k] = s[k][0];
}

__global__ void k_offset_moments_sum(const double* __restrict__ part, int npairs,
                                     double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs * 6) return;
  const int pr = i / 6, k = i % 6;
  double acc = 0.0;
  for (int b = 0; b < kOffsetParts; ++b) acc += part[((size_t)pr * kOffsetParts + b) * 6 + k];
  out[i] = acc;
}

int offset_moments(Context* c, const float* corr, int w, int h, const OffsetPair* d_pairs,
                   int npairs, double* d_out, cudaStream_t st) {
  if (npairs <= 0) return MF_OK;
  DevBuf part;
  MF_TRY(part.alloc(sizeof(double) * 6 * kOffsetParts * (size_t)npairs));
  k_offset_moments<<<dim3(npairs, kOffsetParts), 256, 0, st>>>(corr, w, h, d_pairs,
                                                                part.as<double>());
  k_offset_moments_sum<<<(npairs * 6 + 255) / 256, 256, 0, st>>>(part.as<double>(), npairs,
                                                                 d_out);
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

}  // namespace mf
