// CPU oracle for the Markerfree projection-matching alignment path.
//
// TEST INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's CPU-baseline leg
// use it as the checker.  The product library never links or calls it.
//
// FP32 restatement of the reference (nvcc -O3, no fast-math) with FP64 FFTs in
// place of cuFFT.  Each function names the reference lines it follows; paths are
// relative to the reference project root.  Independent output pixels are spread
// over OpenMP threads; every per-pixel reduction keeps the reference's order.
#include "oc_oracle.hpp"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <stdint.h>

#include <algorithm>
#include <complex>
#include <mutex>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "oc_fft.hpp"

namespace {

const double D2R = 4.0 * atan(1.0) / 180.0;  // Markerfree/src/method/Util.h:33
const float kBig = (float)-1e30;

// The reference evaluates cosf/sinf/expf on the GPU.  The oracle uses the
// correctly rounded value of the same float argument unless a test has
// registered CUDA's own cosf/sinf values for it (oc_trig_set: measured on the
// GPU, not restated).  The two differ in the last place for some arguments, and
// such a difference can move a nearest-neighbour index or a common-region end;
// with the values registered the oracle takes the reference's decisions.
// oc_trig_record collects the arguments a call evaluates, for registering.
struct TrigTable {
  std::unordered_map<uint32_t, std::pair<float, float>> v;  // bits of x -> (cos, sin)
  bool recording = false;
  std::unordered_set<uint32_t> seen;
  std::mutex mu;
};
TrigTable& trig_table() {
  static TrigTable t;
  return t;
}
inline uint32_t fbits(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  return u;
}
inline bool trig_lookup(float x, float* c, float* s) {
  TrigTable& t = trig_table();
  if (t.recording) {
    std::lock_guard<std::mutex> lk(t.mu);
    t.seen.insert(fbits(x));
  }
  if (t.v.empty()) return false;
  auto it = t.v.find(fbits(x));
  if (it == t.v.end()) return false;
  *c = it->second.first;
  *s = it->second.second;
  return true;
}
inline float cosf_cr(float x) {
  float c, s;
  if (trig_lookup(x, &c, &s)) return c;
  return (float)cos((double)x);
}
inline float sinf_cr(float x) {
  float c, s;
  if (trig_lookup(x, &c, &s)) return s;
  return (float)sin((double)x);
}
inline float expf_cr(float x) { return (float)exp((double)x); }

// x*c + yprod + o as nvcc compiles the reference's x*c - y*s + o and x*s + y*c + o:
// the first product fused with the second, then the offset added.
inline float lin2(float x, float c, float yprod, float o) { return std::fmaf(x, c, yprod) + o; }

typedef std::complex<double> cd;

// ---------------------------------------------------------------------------
// Util.cpp:8-20
int frame_idx_from_tilt(int nz, const float* a, float tilt) {
  int idx = 0;
  float fmin = (float)fabs(tilt - a[0]);
  for (int i = 1; i < nz; ++i) {
    float d = (float)fabs(tilt - a[i]);
    if (d >= fmin) continue;
    fmin = d;
    idx = i;
  }
  return idx;
}

// Util.cpp:22-35
int find_ref_index(int nz, const float* a, int z) {
  int i0 = z - 1, i2 = z + 1;
  if (i0 < 0) i0 = z;
  if (i2 >= nz) i2 = z;
  double t0 = fabs(a[i0]), t = fabs(a[z]), t2 = fabs(a[i2]);
  if (t0 < t) return i0;
  if (t2 < t) return i2;
  return z;
}

// ---------------------------------------------------------------------------
// CorrStack.cu:116-140 (deterministic "random" fill for the resampler)
float corr_random(int x, int y, int in_x, int in_y, int in_stride, const float* img) {
  if (x < 0) x = -x;
  if (y < 0) y = -y;
  if (x >= in_x) x = in_x - 1 - (x % in_x);
  if (y >= in_y) y = in_y - 1 - (y % in_y);
  const int win = 51, size = win * win;
  unsigned int next = (unsigned int)(y * in_stride + x);
  for (int i = 0; i < 20; ++i) {
    next = (next * 19u + 57u) % (unsigned int)size;
    int ix = (int)(next % (unsigned int)size) - win / 2 + x;
    if (ix < 0 || ix >= in_x) continue;
    int iy = (int)(next / (unsigned int)win) - win / 2 + y;
    if (iy < 0 || iy >= in_y) continue;
    return img[iy * in_stride + ix];
  }
  return img[y * in_stride + x];
}

// CorrStack.cu:142-179 — one output pixel of the rotate+shift resampler.
// out_x is the unpadded output width (grid width), out_y its height.
inline float corr_pixel(const float* img, int in_x, int in_y, int bx, int y, int out_x, int out_y,
                        float sx, float sy, float cs, float sn, bool random_fill) {
  float ax = (float)bx + 0.5f - (float)out_x * 0.5f;
  float ay = (float)y + 0.5f - (float)out_y * 0.5f;
  // nvcc fuses the first product of each sum in the reference's device code
  float t = std::fmaf(ax, cs, -(ay * sn));
  ay = std::fmaf(ax, sn, ay * cs);
  ax = t;
  ax += (sx + (float)in_x * 0.5f);
  ay += (sy + (float)in_y * 0.5f);
  int ix = (int)(ax + 0.5f);
  int iy = (int)(ay + 0.5f);
  if (ix >= 0 && ix < in_x && iy >= 0 && iy < in_y) return img[iy * in_x + ix];
  if (random_fill) return corr_random(ix, iy, in_x, in_y, in_x, img);
  return kBig;
}

// CorrStack.cu:65-75 / 16-23
void binned_size(int nx, int ny, int bin, int* xb, int* yb) {
  *xb = nx / bin / 2 * 2;
  *yb = ny / bin / 2 * 2;
}

// CorrStack.cu:431-446 — per-row ramp x raised-cosine weighting between 1-D FFTs.
void rweight_rows(float* img, int xb, int yb) {
  int cmp = xb / 2 + 1;
  float fN = 2 * ((float)cmp - 1.0f);
  std::vector<float> fr(cmp);
  for (int x = 0; x < cmp; ++x) {
    float r = (float)x / fN;
    r = 2 * r * std::fmaf(0.45f, cosf_cr(6.2831852f * r), 0.55f);
    fr[x] = r;
  }
#pragma omp parallel
  {
    std::vector<double> row(xb);
    std::vector<cd> spec(cmp);
#pragma omp for schedule(static)
    for (int y = 0; y < yb; ++y) {
      float* p = img + (size_t)y * xb;
      for (int x = 0; x < xb; ++x) row[x] = p[x];
      oc::fft_r2c_1d(row.data(), spec.data(), xb);
      for (int x = 0; x < cmp; ++x) {
        // the kernel rounds each step to float on cuFFT's float spectrum
        float re = (float)spec[x].real(), im = (float)spec[x].imag();
        re /= fN;
        im /= fN;
        re *= fr[x];
        im *= fr[x];
        spec[x] = cd(re, im);
      }
      oc::fft_c2r_1d(spec.data(), row.data(), xb);
      for (int x = 0; x < xb; ++x) p[x] = (float)row[x];
    }
  }
}

// CorrStack.cu:370-397 (mCorrectProj) with Set1/Set2 options.
void correct_proj(const float* proj, int nx, int ny, float shift_x, float shift_y,
                  float tilt_axis_deg, bool only_shift, int bin, bool random_fill, bool rweight,
                  float* out) {
  // CalcAlignedSize never swaps (CorrStack.cu:3-14), so the aligned size is nx x ny.
  int pad_x = (nx / 2 + 1) * 2;
  int out_x = (pad_x / 2 - 1) * 2;  // GCorrPatchShift::SetSizes, CorrStack.cu:204
  int out_y = ny;
  float axis = only_shift ? 0.0f : tilt_axis_deg;
  axis = (float)(axis * D2R);  // CorrStack.cu:376-378
  float cs = cosf_cr(axis), sn = sinf_cr(axis);
  int xb, yb;
  binned_size(nx, ny, bin, &xb, &yb);
  int binx = out_x / xb;  // BinImage::SetupSizes, CorrStack.cu:94-100
  int biny = ny / yb;
  std::vector<float> corr((size_t)out_x * out_y);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < out_y; ++y)
    for (int x = 0; x < out_x; ++x)
      corr[(size_t)y * out_x + x] =
          corr_pixel(proj, nx, ny, x, y, out_x, out_y, shift_x, shift_y, cs, sn, random_fill);
  // mGBinImage (CorrStack.cu:40-63)
#pragma omp parallel for schedule(static)
  for (int y = 0; y < yb; ++y) {
    for (int x = 0; x < xb; ++x) {
      float sum = 0.0f;
      bool bad = false;
      for (int iy = 0; iy < biny && !bad; ++iy) {
        const float* p = &corr[(size_t)(y * biny + iy) * out_x];
        for (int ix = 0; ix < binx; ++ix) {
          float v = p[x * binx + ix];
          if (v < (float)-1e10) {
            bad = true;
            break;
          }
          sum += v;
        }
      }
      out[(size_t)y * xb + x] = bad ? kBig : sum;
    }
  }
  if (rweight) rweight_rows(out, xb, yb);
}

// ---------------------------------------------------------------------------
// CalcReproj.cu:206-259 (FindProjRange)
void find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj, int nproj,
                     int* range) {
  const float ref_range = 20.5f, ref_stretch = 1.2f;
  float tilt = angles[iproj];
  float fcos = (float)cos(tilt * D2R);
  int istart = -1;
  for (int i = 0; i < nz; ++i) {
    if (skip[i]) continue;
    float diff = tilt - angles[i];
    if (fabs(diff) > ref_range) continue;
    float st = (float)(cos(angles[i] * D2R) / fcos);
    if (st > ref_stretch) continue;
    istart = i;
    break;
  }
  int iend = -1;
  // The reference starts this scan at istart even when it is -1; with no
  // neighbour both stay -1 here and the caller reports the error.
  for (int i = (istart < 0 ? 0 : istart); istart >= 0 && i < nz; ++i) {
    if (skip[i]) continue;
    float diff = tilt - angles[i];
    if (fabs(diff) > ref_range) continue;
    float st = (float)(cos(angles[i] * D2R) / fcos);
    if (st > ref_stretch) continue;
    iend = i;
  }
  int np = nproj - 1;
  if ((iend - istart) > np) {
    int zero = frame_idx_from_tilt(nz, angles, 0.0f);
    if (iproj < zero)
      iend = istart + np;
    else
      istart = iend - np;
  }
  range[0] = istart;
  range[1] = iend;
}

// CalcReproj.cu:17-64 (mGBackProj + mDIntProj) and :68-124 (mGForProj),
// driven row by row as in CalcReprojFBP::DoIt (:180-204).
void reproject(const float* corr, int xb, int yb, int nz, const float* angles, int iproj,
               int istart, int iend, int thickness, float* out) {
  (void)nz;
  const float s_fD2R = 0.01745f;
  const int W = 2 * xb, T = thickness;
  const float proj_angle = angles[iproj];
  int nk = iend - istart + 1;
  std::vector<float> bw(nk), bc(nk), bs(nk);
  for (int k = 0; k < nk; ++k) {
    float a = angles[istart + k];
    bw[k] = cosf_cr((proj_angle - a) * s_fD2R);
    float v = a * s_fD2R;
    bc[k] = cosf_cr(v);
    bs[k] = sinf_cr(v);
  }
  const float fcos = (float)cos(D2R * proj_angle);
  const float fsin = (float)sin(D2R * proj_angle);
  const int ray_len = (int)((float)T / fcos + 0.5f);
  const size_t pix = (size_t)xb * yb;
#pragma omp parallel
  {
    std::vector<float> slab((size_t)W * T);
    std::vector<float> lane_sum(512);
    std::vector<int> lane_cnt(512);
#pragma omp for schedule(dynamic, 4)
    for (int y = 0; y < yb; ++y) {
      // back-projection of one xz slice
      const float cent_x = (float)xb * 0.5f;
      const int iend_x = xb - 1;
      for (int iz = 0; iz < T; ++iz) {
        float fz = (float)iz + 0.5f - (float)T * 0.5f;
        for (int ix = 0; ix < W; ++ix) {
          float fx = (float)ix + 0.5f - (float)W * 0.5f;
          float fint = 0.0f, fcount = 0.0f;
          for (int k = 0; k < nk; ++k) {
            float v = std::fmaf(fx, bc[k], fz * bs[k]) + cent_x;
            if (v < 0 || v > iend_x) continue;
            const float* row = corr + (size_t)(istart + k) * pix + (size_t)y * xb;
            float val = row[(int)v];
            if (val < (float)-1e10) val = kBig;
            if (val < (float)-1e20) continue;
            fint = std::fmaf(val * bc[k], bw[k], fint);
            fcount += bw[k];
          }
          slab[(size_t)iz * W + ix] = (fcount < 0.001f) ? kBig : fint / fcount;
        }
      }
      // forward projection: 512 lanes per ray, then a tree reduction
      const int iendx = W - 1, iendz = T - 1;
      const int nseg = ray_len / 512 + 1;
      for (int bx = 0; bx < xb; ++bx) {
        float fxp = (float)bx + 0.5f - (float)xb * 0.5f;
        float tx = std::fmaf(fxp, fcos, (float)W * 0.5f);
        float tz = std::fmaf(fxp, fsin, (float)T * 0.5f);
        float zst = -fxp * fsin / fcos - 0.5f * (float)ray_len;
        for (int t = 0; t < 512; ++t) {
          float s = 0.0f;
          int c = 0;
          for (int seg = 0; seg < nseg; ++seg) {
            int j = seg * 512 + t;
            if (j >= ray_len) continue;
            float fz = (float)j + zst;
            float fx = std::fmaf(-fz, fsin, tx);
            fz = std::fmaf(fz, fcos, tz);
            if (fx >= 0 && fx < iendx && fz >= 0 && fz < iendz) {
              float v = slab[(size_t)(int)fz * W + (int)fx];
              if (v >= (float)-1e10) {
                s += v;
                c += 1;
              }
            }
          }
          lane_sum[t] = s;
          lane_cnt[t] = c;
        }
        for (int h = 256; h > 0; h /= 2)
          for (int t = 0; t < h; ++t) {
            lane_sum[t] += lane_sum[t + h];
            lane_cnt[t] += lane_cnt[t + h];
          }
        float r;
        if ((float)lane_cnt[0] < 0.8f * (float)ray_len)
          r = kBig;
        else
          r = lane_sum[0] / (float)lane_cnt[0];
        out[(size_t)y * xb + bx] = r;
      }
    }
  }
}

// The same re-projection with every value accumulated in FP64 (back-projection
// sums, slab cells, ray sums and means) and the same index decisions, taken in
// FP32 exactly as above: the reference's discrete geometry with exact-as-possible
// arithmetic, against which the FP32, FP16 and BF16 paths state their errors.
void reproject_f64(const float* corr, int xb, int yb, int nz, const float* angles, int iproj,
                   int istart, int iend, int thickness, double* out) {
  (void)nz;
  const float s_fD2R = 0.01745f;
  const int W = 2 * xb, T = thickness;
  const float proj_angle = angles[iproj];
  int nk = iend - istart + 1;
  std::vector<float> bw(nk), bc(nk), bs(nk);
  for (int k = 0; k < nk; ++k) {
    float a = angles[istart + k];
    bw[k] = cosf_cr((proj_angle - a) * s_fD2R);
    float v = a * s_fD2R;
    bc[k] = cosf_cr(v);
    bs[k] = sinf_cr(v);
  }
  const float fcos = (float)cos(D2R * proj_angle);
  const float fsin = (float)sin(D2R * proj_angle);
  const int ray_len = (int)((float)T / fcos + 0.5f);
  const size_t pix = (size_t)xb * yb;
#pragma omp parallel
  {
    std::vector<double> slab((size_t)W * T);
    std::vector<double> lane_sum(512);
    std::vector<int> lane_cnt(512);
#pragma omp for schedule(dynamic, 4)
    for (int y = 0; y < yb; ++y) {
      // back-projection of one xz slice
      const float cent_x = (float)xb * 0.5f;
      const int iend_x = xb - 1;
      for (int iz = 0; iz < T; ++iz) {
        float fz = (float)iz + 0.5f - (float)T * 0.5f;
        for (int ix = 0; ix < W; ++ix) {
          float fx = (float)ix + 0.5f - (float)W * 0.5f;
          double fint = 0.0, fcount = 0.0;
          for (int k = 0; k < nk; ++k) {
            float v = std::fmaf(fx, bc[k], fz * bs[k]) + cent_x;
            if (v < 0 || v > iend_x) continue;
            const float* row = corr + (size_t)(istart + k) * pix + (size_t)y * xb;
            float val = row[(int)v];
            if (val < (float)-1e10) val = kBig;
            if (val < (float)-1e20) continue;
            fint += (double)val * bc[k] * bw[k];
            fcount += bw[k];
          }
          slab[(size_t)iz * W + ix] = (fcount < 0.001) ? (double)kBig : fint / fcount;
        }
      }
      // forward projection: 512 lanes per ray, then a tree reduction
      const int iendx = W - 1, iendz = T - 1;
      const int nseg = ray_len / 512 + 1;
      for (int bx = 0; bx < xb; ++bx) {
        float fxp = (float)bx + 0.5f - (float)xb * 0.5f;
        float tx = std::fmaf(fxp, fcos, (float)W * 0.5f);
        float tz = std::fmaf(fxp, fsin, (float)T * 0.5f);
        float zst = -fxp * fsin / fcos - 0.5f * (float)ray_len;
        for (int t = 0; t < 512; ++t) {
          double s = 0.0;
          int c = 0;
          for (int seg = 0; seg < nseg; ++seg) {
            int j = seg * 512 + t;
            if (j >= ray_len) continue;
            float fz = (float)j + zst;
            float fx = std::fmaf(-fz, fsin, tx);
            fz = std::fmaf(fz, fcos, tz);
            if (fx >= 0 && fx < iendx && fz >= 0 && fz < iendz) {
              double v = slab[(size_t)(int)fz * W + (int)fx];
              if (v >= -1e10) {
                s += v;
                c += 1;
              }
            }
          }
          lane_sum[t] = s;
          lane_cnt[t] = c;
        }
        for (int h = 256; h > 0; h /= 2)
          for (int t = 0; t < h; ++t) {
            lane_sum[t] += lane_sum[t + h];
            lane_cnt[t] += lane_cnt[t + h];
          }
        double r;
        if ((float)lane_cnt[0] < 0.8f * (float)ray_len)
          r = kBig;
        else
          r = lane_sum[0] / (double)lane_cnt[0];
        out[(size_t)y * xb + bx] = r;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// CalcCC.cu:48-92 (CalcMoment: masked sum / (w*h)); accumulated in FP64 here.
float calc_moment(const float* img, int w, int h, int stride, int e) {
  double s = 0.0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float v = img[(size_t)y * stride + x];
      if (v < (float)-1e10) continue;
      float ev = v;
      for (int i = 1; i < e; ++i) ev *= v;
      s += ev;
    }
  return (float)(s / ((double)w * h));
}

// CalcCC.cu:137-147
void norm2d(float* img, int w, int h, int stride, float mean, float sd) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float& v = img[(size_t)y * stride + x];
      if (v < (float)-1e10) continue;
      v = (v - mean) / sd;
    }
}

// CalcCC.cu:173-195
void round_edge(float* img, int w, int h, int stride, float cx, float cy, float sx, float sy,
                float power) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float& v = img[(size_t)y * stride + x];
      if (v < (float)-1e10) {
        v = 0.0f;
        continue;
      }
      float fx = 2 * fabsf((float)x - cx) / sx;
      float fy = 2 * fabsf((float)y - cy) / sy;
      float fr = sqrtf(std::fmaf(fx, fx, fy * fy));
      if (fr >= 1.0f) {
        v = 0.0f;
        continue;
      }
      fr = 0.5f * (1 - cosf_cr(3.1415926f * fr));
      fr = 1.0f - powf(fr, power);
      v = v * fr;
    }
}

// 2-D R2C of a padded image (rows of `stride` floats, first nx used), with an
// optional 1/N scale (Cufft1&2.cu:27-62 with GMultiplyFactor).
std::vector<cd> fwd2d(const float* img, int nx, int ny, int stride, bool norm) {
  std::vector<double> buf((size_t)nx * ny);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) buf[(size_t)y * nx + x] = img[(size_t)y * stride + x];
  int cx = nx / 2 + 1;
  std::vector<cd> spec((size_t)cx * ny);
  oc::fft_r2c_2d(buf.data(), nx, spec.data(), nx, ny);
  for (auto& c : spec) c = cd((float)c.real(), (float)c.imag());
  if (norm) {
    float f = (float)(1.0 / ((cx - 1) * 2) / ny);
    for (auto& c : spec) c = cd((float)c.real() * f, (float)c.imag() * f);
  }
  return spec;
}

// CalcCC.cu:95-135 (GConv, GWiener, GCenterOrigin) then the C2R of
// ProjAlign.cpp:314-323 / CalcCC.cu:366-379.  Returns the real map (ny x nx).
std::vector<float> xcorr_map(const std::vector<cd>& ref, std::vector<cd> img, int nx, int ny,
                             float bfactor) {
  int cx = nx / 2 + 1;
  for (int y = 0; y < ny; ++y) {
    for (int x = 0; x < cx; ++x) {
      size_t i = (size_t)y * cx + x;
      float ar = (float)ref[i].real(), ai = (float)ref[i].imag();
      float br = (float)img[i].real(), bi = (float)img[i].imag();
      float re = std::fmaf(ar, br, ai * bi);
      float im = std::fmaf(ar, bi, -(ai * br));
      // Wiener / B-factor
      int yy = y;
      if (yy > (ny / 2)) yy -= ny;
      float fnx = 2.0f * (float)(cx - 1);
      float filt = -2.0f * bfactor / std::fmaf(fnx, fnx, (float)(ny * ny));
      filt = expf_cr(filt * (float)((unsigned)(x * x) + (unsigned)(yy * yy)));
      float amp = sqrtf(std::fmaf(re, re, im * im));
      filt /= sqrtf(amp + 0.01f);
      re *= filt;
      im *= filt;
      // centre the origin
      int sgn = ((x + y) % 2 == 0) ? 1 : -1;
      re *= sgn;
      im *= sgn;
      img[i] = cd(re, im);
    }
  }
  std::vector<double> outd((size_t)nx * ny);
  oc::fft_c2r_2d(img.data(), outd.data(), nx, nx, ny);
  std::vector<float> out((size_t)nx * ny);
  for (size_t i = 0; i < out.size(); ++i) out[i] = (float)outd[i];
  return out;
}

// ProjAlign.cpp:325-375 (PAFindPeak); map is dense ny x nx.
float pa_find_peak(const std::vector<float>& m, int nx, int ny, float* shift) {
  float fpeak = (float)-1e20;
  int px = 0, py = 0;
  int sx = nx / 20, sy = ny / 20;
  if (sx < 3) sx = 3;
  if (sy < 3) sy = 3;
  int ex = nx - sx, ey = ny - sy;
  for (int y = sy; y < ey; ++y)
    for (int x = sx; x < ex; ++x) {
      float v = m[(size_t)y * nx + x];
      if (fpeak >= v) continue;
      px = x;
      py = y;
      fpeak = v;
    }
  size_t ic = (size_t)py * nx + px;
  double a = (m[ic + 1] + m[ic - 1]) * 0.5 - m[ic];
  double b = (m[ic + 1] - m[ic - 1]) * 0.5;
  double c = (m[ic + nx] + m[ic - nx]) * 0.5 - m[ic];
  double d = (m[ic + nx] - m[ic - nx]) * 0.5;
  double dx = -b / (2 * a + 1e-30);
  double dy = -d / (2 * c + 1e-30);
  if (fabs(dx) > 1) dx = 0;
  if (fabs(dy) > 1) dy = 0;
  float pkx = (float)(px + dx), pky = (float)(py + dy);
  shift[0] = pkx - nx / 2;
  shift[1] = pky - ny / 2;
  return (float)(a * dx * dx + b * dx + c * dy * dy + d * dy + m[ic]);
}

// ProjAlign.cpp:243-312 (MeaAlignProj with PANorm / GetCentral)
float measure_shift(const float* reproj, const float* proj, int xb, int yb, float* shift) {
  int pad = (xb / 2 + 1) * 2;
  auto panorm = [&](const float* img) {
    std::vector<float> p((size_t)pad * yb, 0.0f);
    for (int y = 0; y < yb; ++y) memcpy(&p[(size_t)y * pad], img + (size_t)y * xb, xb * 4);
    int w = (pad / 2 - 1) * 2;
    float mean = calc_moment(p.data(), w, yb, pad, 1);
    norm2d(p.data(), w, yb, pad, mean, 1.0f);
    float cx = (float)((pad / 2 - 1) * 2) * 0.5f, cy = (float)yb * 0.5f;
    round_edge(p.data(), w, yb, pad, cx, cy, (float)pad, (float)yb, 4.0f);
    return p;
  };
  std::vector<float> r = panorm(reproj), m = panorm(proj);
  auto R = fwd2d(r.data(), xb, yb, pad, false);
  auto I = fwd2d(m.data(), xb, yb, pad, false);
  std::vector<float> map = xcorr_map(R, I, xb, yb, 500.0f);
  return pa_find_peak(map, xb, yb, shift);
}

// RotShift (ProjAlign.cpp:448-457)
void rot_shift(const float* in, float angle, float* out) {
  float c = (float)cos(angle * D2R), s = (float)sin(angle * D2R);
  float sx = in[0] * c - in[1] * s;
  float sy = in[0] * s + in[1] * c;
  out[0] = sx;
  out[1] = sy;
}

}  // namespace

// ===========================================================================
extern "C" {

// Register cos/sin values for float arguments (replacing earlier ones); n = 0 clears.
void oc_trig_set(int n, const float* x, const float* c, const float* s) {
  TrigTable& t = trig_table();
  if (n <= 0) t.v.clear();
  for (int i = 0; i < n; ++i) t.v[fbits(x[i])] = std::make_pair(c[i], s[i]);
}

// on = 1: start collecting the arguments cosf/sinf are evaluated at; on = 0: stop.
void oc_trig_record(int on) {
  TrigTable& t = trig_table();
  if (on) t.seen.clear();
  t.recording = on != 0;
}

// The collected arguments: returns their number, writes at most `max`.
int oc_trig_recorded(float* out, int max) {
  TrigTable& t = trig_table();
  int n = 0;
  for (uint32_t u : t.seen) {
    if (n < max) memcpy(out + n, &u, 4);
    ++n;
  }
  return n;
}

int oc_frame_idx_from_tilt(int nz, const float* a, float t) { return frame_idx_from_tilt(nz, a, t); }
int oc_find_ref_index(int nz, const float* a, int z) { return find_ref_index(nz, a, z); }

void oc_binned_size(int nx, int ny, int bin, int* xb, int* yb) { binned_size(nx, ny, bin, xb, yb); }

void oc_correct_proj(const float* proj, int nx, int ny, float sx, float sy, float axis,
                     int only_shift, int bin, int random_fill, int rweight, float* out) {
  correct_proj(proj, nx, ny, sx, sy, axis, only_shift != 0, bin, random_fill != 0, rweight != 0,
               out);
}

void oc_find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                        int nproj, int* range2) {
  find_proj_range(angles, nz, skip, iproj, nproj, range2);
}

void oc_reproject(const float* corr, int xb, int yb, int nz, const float* angles, int iproj,
                  int istart, int iend, int thickness, float* out) {
  reproject(corr, xb, yb, nz, angles, iproj, istart, iend, thickness, out);
}

void oc_reproject_f64(const float* corr, int xb, int yb, int nz, const float* angles, int iproj,
                      int istart, int iend, int thickness, double* out) {
  reproject_f64(corr, xb, yb, nz, angles, iproj, istart, iend, thickness, out);
}

void oc_measure_shift(const float* reproj, const float* proj, int xb, int yb, float* shift2,
                      float* peak) {
  float p = measure_shift(reproj, proj, xb, yb, shift2);
  if (peak) *peak = p;
}

// ---------------------------------------------------------------------------
// Preprocess.cu:103-250
void oc_preprocess(const float* raw, int nx, int ny, int nz, const float* angles, float* out) {
  size_t pix = (size_t)nx * ny;
  bool rev = angles[0] > angles[1];
  float stack_min = (float)1e30;
  for (int a = 0; a < nz; ++a) {
    int i = rev ? nz - 1 - a : a;
    memcpy(out + (size_t)i * pix, raw + (size_t)a * pix, pix * 4);
    float mn = (float)1e20;
    for (size_t k = 0; k < pix; ++k) {
      float v = raw[(size_t)a * pix + k];
      if (v < (float)-1e10) continue;
      mn = fminf(mn, v);
    }
    if (stack_min > mn) stack_min = mn;
  }
  if (!(stack_min >= 0)) {
    for (size_t k = 0; k < pix * nz; ++k) {
      if (out[k] < (float)-1e10) continue;
      out[k] -= stack_min;
    }
  }
  // MassNormalization: central 4/6 box; the zero tilt is looked up in the
  // angles as read from the file (not reversed), as the reference does.
  int sx0 = nx * 1 / 6, sy0 = ny * 1 / 6, w = nx * 4 / 6, h = ny * 4 / 6;
  std::vector<float> mean(nz);
  for (int i = 0; i < nz; ++i) {
    double dm = 0.0;
    int cnt = 0;
    const float* f = out + (size_t)i * pix;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        float v = f[(size_t)(y + sy0) * nx + sx0 + x];
        if (v <= (float)-1e20) continue;
        dm += v;
        cnt++;
      }
    mean[i] = cnt == 0 ? 0.0f : (float)(dm / cnt);
  }
  int zero = frame_idx_from_tilt(nz, angles, 0.0f);
  float ref = mean[zero];
  if (ref > 1000.0f) ref = 1000.0f;
  for (int i = 0; i < nz; ++i) {
    float sc = ref / (mean[i] + 0.00001f);
    float* f = out + (size_t)i * pix;
    for (size_t k = 0; k < pix; ++k) {
      if (f[k] <= (float)-1e20) continue;
      f[k] *= sc;
    }
  }
}

// ---------------------------------------------------------------------------
// ProjAlign (ProjAlign.cpp:48-579), one instance per mProjAlign call.
struct oc_projalign {
  const float* stack;
  int nx, ny, nz;
  std::vector<float> angles;
  oc_param* param;
  float z0, x0;
  int bin, xb, yb, thick, nproj;
  std::vector<float> corr;  // nz x yb x xb
  std::vector<unsigned char> skip;
  std::vector<float> reproj;
  std::vector<float> meas;  // per tilt: measured shift (un-binned px) of the last pass
  bool f64 = false;         // re-project with every value accumulated in FP64
  std::vector<double> reproj64;
};

static void pa_correct(oc_projalign* pa, int i) {
  size_t pix = (size_t)pa->nx * pa->ny;
  correct_proj(pa->stack + i * pix, pa->nx, pa->ny, pa->param->shift_x[i], pa->param->shift_y[i],
               pa->param->rotate[i], false, pa->bin, true, true,
               pa->corr.data() + (size_t)i * pa->xb * pa->yb);
}

// CalcZInducedShift (ProjAlign.cpp:553-561)
static void z_induced(oc_projalign* pa, int f, float* s) {
  s[0] = s[1] = 0.0f;
  if (pa->z0 == 0) return;
  float t = (float)(pa->angles[f] * D2R);
  s[0] = (float)(-pa->z0 * sin(t));
  rot_shift(s, pa->param->rotate[f], s);
}

oc_projalign* oc_projalign_create(const float* stack, int nx, int ny, int nz, const float* angles,
                                  oc_param* param, float zshift, int align_z, int nproj) {
  oc_projalign* pa = new oc_projalign();
  pa->stack = stack;
  pa->nx = nx;
  pa->ny = ny;
  pa->nz = nz;
  pa->angles.assign(angles, angles + nz);
  pa->param = param;
  pa->z0 = zshift;
  pa->x0 = 0;
  pa->nproj = nproj;
  int bx = (int)((float)nx / 2048.0f + 0.5f), by = (int)((float)ny / 2048.0f + 0.5f);
  pa->bin = bx > by ? bx : by;
  if (pa->bin < 1) pa->bin = 1;
  binned_size(nx, ny, pa->bin, &pa->xb, &pa->yb);
  pa->thick = align_z / pa->bin / 2 * 2;
  pa->corr.assign((size_t)nz * pa->xb * pa->yb, 0.0f);
  pa->skip.assign(nz, 1);
  pa->reproj.assign((size_t)pa->xb * pa->yb, 0.0f);
  pa->meas.assign((size_t)2 * nz, 0.0f);
  return pa;
}

float oc_projalign_z0(const oc_projalign* pa) { return pa->z0; }
void oc_projalign_measured(const oc_projalign* pa, float* xy) {
  for (int i = 0; i < 2 * pa->nz; ++i) xy[i] = pa->meas[i];
}
int oc_projalign_bin(const oc_projalign* pa) { return pa->bin; }
void oc_projalign_destroy(oc_projalign* pa) { delete pa; }

// on = 1: later passes re-project in FP64 (reproject_f64) instead of FP32.
void oc_projalign_set_f64(oc_projalign* pa, int on) { pa->f64 = on != 0; }

// ProjAlign.cpp:133-179 (DoItBin) + 181-241 (ClacAlignProj) + 459-501.
float oc_projalign_doit(oc_projalign* pa) {
  int nz = pa->nz;
  for (int i = 0; i < nz; ++i) pa_correct(pa, i);
  // FitRotCenterZ (ProjAlign.cpp:459-486; the uninitialised dA is taken as 0)
  {
    int zt = frame_idx_from_tilt(nz, pa->angles.data(), 0.0f);
    float s0[2] = {pa->param->shift_x[zt], pa->param->shift_y[zt]};
    rot_shift(s0, -pa->param->rotate[zt], s0);
    float cent0 = (float)(s0[0] / cos(pa->angles[zt] * D2R));
    double dA = 0.0, dB = 0.0;
    for (int i = 0; i < nz; ++i) {
      float raw[2] = {pa->param->shift_x[i], pa->param->shift_y[i]}, rs[2];
      rot_shift(raw, -pa->param->rotate[i], rs);
      double ds = sin(pa->angles[i] * D2R), dc = cos(pa->angles[i] * D2R);
      dA += (cent0 * dc - rs[0]) * ds;
      dB += ds * ds;
    }
    pa->z0 = (float)(dA / (dB + 1e-30));
  }
  // RemoveOffsetZ(-1) (ProjAlign.cpp:488-501)
  int zt = frame_idx_from_tilt(nz, pa->angles.data(), 0.0f);
  if (pa->z0 != 0) {
    for (int i = 0; i < nz; ++i) {
      if (i == zt) continue;
      float s[2];
      z_induced(pa, i, s);
      pa->param->shift_x[i] += s[0] * -1.0f;
      pa->param->shift_y[i] += s[1] * -1.0f;
    }
  }
  for (int i = 0; i < nz; ++i) pa->skip[i] = 1;
  pa->skip[zt] = 0;
  float max_err = (float)-1e20;
  size_t bpix = (size_t)pa->xb * pa->yb;
  for (int i = 1; i < nz; ++i) {
    for (int side = 0; side < 2; ++side) {
      int ip = side == 0 ? zt + i : zt - i;
      if (ip >= nz || ip < 0) continue;
      int rg[2];
      find_proj_range(pa->angles.data(), nz, pa->skip.data(), ip, pa->nproj, rg);
      if (rg[0] < 0 || rg[1] < 0) {
        fprintf(stderr, "oracle: no neighbour in range for tilt %d\n", ip);
        return -1.0f;
      }
      if (pa->f64) {  // FP64 re-projection, rounded once to the FP32 image
        pa->reproj64.resize(pa->reproj.size());
        reproject_f64(pa->corr.data(), pa->xb, pa->yb, nz, pa->angles.data(), ip, rg[0], rg[1],
                      pa->thick, pa->reproj64.data());
        for (size_t q = 0; q < pa->reproj.size(); ++q) pa->reproj[q] = (float)pa->reproj64[q];
      } else {
        reproject(pa->corr.data(), pa->xb, pa->yb, nz, pa->angles.data(), ip, rg[0], rg[1],
                  pa->thick, pa->reproj.data());
      }
      float sh[2];
      measure_shift(pa->reproj.data(), pa->corr.data() + ip * bpix, pa->xb, pa->yb, sh);
      float af[2];
      float bx = (float)pa->nx / (float)pa->xb, by = (float)pa->ny / (float)pa->yb;
      af[0] = sh[0] * bx;
      af[1] = sh[1] * by;
      pa->meas[2 * ip] = af[0];
      pa->meas[2 * ip + 1] = af[1];
      float fs = af[0] * af[0] + af[1] * af[1];
      fs = (float)sqrt(fs);
      rot_shift(af, pa->param->rotate[ip], af);
      float ind[2];
      z_induced(pa, ip, ind);
      af[0] += ind[0];
      af[1] += ind[1];
      // CalcXInducedShift is zero: m_fX0 stays 0 (FitRotCenterX is never called).
      pa->param->shift_x[ip] += af[0];
      pa->param->shift_y[ip] += af[1];
      pa_correct(pa, ip);
      pa->skip[ip] = 0;
      if (fs > max_err) max_err = fs;
    }
  }
  return max_err;
}

// ---------------------------------------------------------------------------
// Rotate.cu:292-572 (CalcTIltAxis::DoIt)
float oc_tilt_axis_scores(const float* stack, int nx, int ny, int nz, const float* angles,
                          oc_param* param, float range, int num, float* scores_out) {
  int zt = frame_idx_from_tilt(nz, angles, 0.0f);
  float axis0 = param->rotate[zt];
  float step = range / (num - 1);
  std::vector<float> rot(num);
  rot[0] = axis0 - step * num / 2;
  for (int i = 1; i < num; ++i) rot[i] = rot[i - 1] + step;
  float fmin_size = (float)1e20;
  for (int i = 0; i < num; ++i) {
    float fs = (float)fabs(sin(D2R * rot[i]));
    float fc = (float)fabs(cos(D2R * rot[i]));
    float s1 = (float)nx / (fs + 0.000001f);
    float s2 = (float)ny / (fc + 0.000001f);
    if (fmin_size > s1) fmin_size = s1;
    if (fmin_size > s2) fmin_size = s2;
  }
  int L = (int)fmin_size;
  L = L / 2 * 2 - 100;
  int cmp = L / 2 + 1;
  // common region (GCalcCommonRegion, :9-40); unset entries stay 0 here
  std::vector<int> region((size_t)num * L * 2, 0);
  {
    float sx = param->shift_x[zt], sy = param->shift_y[zt];
    for (int b = 0; b < num; ++b) {
      float a = rot[b] * 3.1415926f / 180.0f;
      float fs = sinf_cr(a), fc = cosf_cr(a);
      int half = L / 2;
      float ox = (float)nx * 0.5f + sx, oy = (float)ny * 0.5f + sy;
      for (int y = 0; y < L; ++y) {
        size_t i = (size_t)b * L + y;
        float fy = (float)y - (float)L * 0.5f;
        for (int x = 1; x < half; ++x) {
          float oxx = lin2((float)-x, fc, -(fy * fs), ox);
          float oyy = lin2((float)-x, fs, fy * fc, oy);
          if (oxx < 0 || oxx >= nx) break;
          if (oyy < 0 || oyy >= ny) break;
          region[2 * i] = -x;
        }
        for (int x = 1; x < half; ++x) {
          float oxx = lin2((float)x, fc, -(fy * fs), ox);
          float oyy = lin2((float)x, fs, fy * fc, oy);
          if (oxx < 0 || oxx >= nx) break;
          if (oyy < 0 || oyy >= ny) break;
          region[2 * i + 1] = x;
        }
      }
    }
  }
  // Radon + per-line mean/window + 1-D FFT (GRadon :42-95, FFT1d :430-451)
  std::vector<cd> planes((size_t)nz * num * cmp);
  size_t pix = (size_t)nx * ny;
  for (int z = 0; z < nz; ++z) {
    float sx = param->shift_x[z], sy = param->shift_y[z];
    float fcos_t = (float)cos(angles[z] * D2R);
    const float* proj = stack + z * pix;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < num; ++b) {
      std::vector<float> line(L + 2);
      float a = rot[b] * 3.1415926f / 180.0f;
      float fsr = sinf_cr(a), fcr = cosf_cr(a);
      float ox = (float)nx * 0.5f + sx, oy = (float)ny * 0.5f + sy;
      for (int y = 0; y < L; ++y) {
        float fy = (float)y - (float)L * 0.5f;
        size_t i = (size_t)b * L + y;
        float sum = 0.0f;
        int cnt = 0;
        int left = (int)std::fmaf((float)region[2 * i], fcos_t, 0.5f);
        for (int x = left; x < 0; ++x) {
          float oxx = lin2((float)x, fcr, -(fy * fsr), ox);
          float oyy = lin2((float)x, fsr, fy * fcr, oy);
          if (oxx < 0 || oxx >= nx) continue;
          if (oyy < 0 || oyy >= ny) continue;
          float v = proj[(size_t)(int)oyy * nx + (int)oxx];
          if (v < 0) continue;
          sum += v;
          cnt++;
        }
        int right = (int)std::fmaf((float)region[2 * i + 1], fcos_t, 0.5f);
        for (int x = 0; x < right; ++x) {
          float oxx = lin2((float)x, fcr, -(fy * fsr), ox);
          float oyy = lin2((float)x, fsr, fy * fcr, oy);
          if (oxx < 0 || oxx >= nx) continue;
          if (oyy < 0 || oyy >= ny) continue;
          float v = proj[(size_t)(int)oyy * nx + (int)oxx];
          if (v < 0) continue;
          sum += v;
          cnt++;
        }
        line[y] = cnt == 0 ? kBig : sum / cnt;
      }
      // GCalcMean (:138-182)
      double msum = 0.0;
      int mcnt = 0;
      for (int y = 0; y < L; ++y)
        if (line[y] > (float)-1e10) {
          msum += line[y];
          mcnt++;
        }
      float mean = mcnt == 0 ? 0.0f : (float)(msum / mcnt);
      // GRemoveMean (:185-198)
      std::vector<double> ld(L);
      for (int y = 0; y < L; ++y) {
        float v = line[y];
        if (v < 0)
          v = 0.0f;
        else
          v -= mean;
        float half = 0.5f * (float)L;
        float fr = fabsf((float)y - half) / half;
        fr = 0.5f * (1 - cosf_cr((float)(3.14159 * fr)));
        fr = 1.0f - powf(fr, 100.0f);
        v *= (fr * fr);
        ld[y] = v;
      }
      std::vector<cd> spec(cmp);
      oc::fft_r2c_1d(ld.data(), spec.data(), L);
      for (int k = 0; k < cmp; ++k)
        planes[((size_t)z * num + b) * cmp + k] = cd((float)spec[k].real(), (float)spec[k].imag());
    }
  }
  // findTiltAxis / CalcScore / GCC1d (:468-602)
  std::vector<float> score(num);
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < num; ++b) {
    std::vector<std::complex<float>> sum(cmp, std::complex<float>(0, 0));
    for (int z = 0; z < nz; ++z)
      for (int k = 0; k < cmp; ++k) {
        cd v = planes[((size_t)z * num + b) * cmp + k];
        sum[k] = std::complex<float>(sum[k].real() * 1.0f + (float)v.real() * 1.0f,
                                     sum[k].imag() * 1.0f + (float)v.imag() * 1.0f);
      }
    float ccsum = 0.0f;
    for (int z = 0; z < nz; ++z) {
      double cc = 0.0, sd = 0.0;
      for (int k = 1; k < cmp; ++k) {
        cd v = planes[((size_t)z * num + b) * cmp + k];
        float lr = (float)v.real(), li = (float)v.imag();
        float rr = sum[k].real() * 1.0f + lr * -1.0f;
        float ri = sum[k].imag() * 1.0f + li * -1.0f;
        float f = (float)k / (2.0f * (float)(cmp - 1));
        f = expf_cr(-2.0f * 10.0f * f * f);
        float a1 = sqrtf(std::fmaf(rr, rr, ri * ri)), a2 = sqrtf(std::fmaf(lr, lr, li * li));
        float c = std::fmaf(lr, rr, li * ri) * f / std::fmaf(a1, a2, (float)1e-20);
        cc += c;
        sd += f;
      }
      ccsum += (float)cc / (float)sd;
    }
    score[b] = ccsum / nz;
  }
  if (scores_out)
    for (int b = 0; b < num; ++b) scores_out[b] = score[b];
  int best = 0;
  float bs = 0.0f;
  for (int b = 0; b < num; ++b)
    if (bs < score[b]) {
      bs = score[b];
      best = b;
    }
  float axis = rot[best];
  if (axis < -45 && param->rotate[0] == 0) axis += 180.0f;
  if (axis > 135) axis -= 180.0f;
  for (int i = 0; i < nz; ++i) param->rotate[i] = axis;
  return axis;
}

float oc_tilt_axis(const float* stack, int nx, int ny, int nz, const float* angles,
                   oc_param* param, float range, int num) {
  return oc_tilt_axis_scores(stack, nx, ny, nz, angles, param, range, num, nullptr);
}

// ---------------------------------------------------------------------------
// CalcCC.cu:8-46, 149-171, 318-345 (stretch about the tilt axis)
static void stretch_matrix(double dstretch, double tilt_axis, float* m) {
  double d2t = 2 * D2R * tilt_axis;
  double s2 = sin(d2t), c2 = cos(d2t);
  double P = 0.5 * (dstretch + 1), M = 0.5 * (dstretch - 1);
  float a0 = (float)(P + M * c2), a1 = (float)(1 * M * s2), a2 = (float)(P - M * c2);
  float det = a0 * a2 - a1 * a1;
  m[0] = a2 / det;
  m[1] = -a1 / det;
  m[2] = a0 / det;
}

static float stretch_random(float X, float Y, int width, int height, int grid_x,
                            const float* in) {
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

// GStretchRandom over a grid of `gw` columns; rows of `stride` floats.
static void stretch(const float* in, int gw, int h, int stride, const float* m, float* out,
                    bool randfill) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < gw; ++x) {
      float X = (float)x - 0.5f * (float)gw + 0.5f;
      float Y = (float)((double)y - 0.5 * h + 0.5f);
      float buf = X * m[0] + Y * m[1];
      Y = X * m[1] + Y * m[2] + 0.5f * (float)h - 0.5f;
      X = buf + 0.5f * (float)gw - 0.5f;
      float v;
      if (X >= 0 && X < gw - 1 && Y >= 0 && Y < h - 1) {
        int ix = (int)X, iy = (int)Y;
        size_t i = (size_t)iy * stride + ix;
        float fx = X - ix, fy = Y - iy;
        float f2 = 1.0f - fx, f3 = 1.0f - fy;
        v = in[i] * f2 * f3 + in[i + 1] * fx * f3 + in[i + stride] * f2 * fy +
            in[i + stride + 1] * fx * fy;
      } else if (randfill) {
        v = stretch_random(X, Y, stride, h, gw, in);
      } else {
        v = kBig;
      }
      out[(size_t)y * stride + x] = v;
    }
}

// Transform (Transform.cpp:24-157)
struct oc_transform {
  const float* stack;
  int nx, ny, nz, bin, xb, yb;
  std::vector<float> angles;
  oc_param* param;
  std::vector<float> pshx, pshy, meas_x, meas_y;
};

oc_transform* oc_transform_create(const float* stack, int nx, int ny, int nz, const float* angles,
                                  oc_param* param) {
  oc_transform* t = new oc_transform();
  t->stack = stack;
  t->nx = nx;
  t->ny = ny;
  t->nz = nz;
  t->angles.assign(angles, angles + nz);
  t->param = param;
  t->pshx.assign(nz, 0.0f);
  t->pshy.assign(nz, 0.0f);
  t->meas_x.assign(nz, 0.0f);
  t->meas_y.assign(nz, 0.0f);
  int bx = (int)((float)nx / 1024.0f + 0.1f), by = (int)((float)ny / 1024.0f + 0.1f);
  t->bin = bx > by ? bx : by;
  if (t->bin < 1) t->bin = 1;
  binned_size(nx, ny, t->bin, &t->xb, &t->yb);
  return t;
}

void oc_transform_destroy(oc_transform* t) { delete t; }

// Per-image shifts measured by the last oc_transform_doit (before UpdateShift
// makes them relative), i.e. the values the reference prints as "Image %d shift".
void oc_transform_measured(const oc_transform* t, float* x, float* y) {
  for (int i = 0; i < t->nz; ++i) {
    x[i] = t->meas_x[i];
    y[i] = t->meas_y[i];
  }
}

// CalcCC::DoIt (CalcCC.cu:237-271) + FindPeak (:381-435); returns shift (binned px).
static void stretch_cc(const float* ref, const float* img, int xb, int yb, float ref_tilt,
                       float tilt, float axis, float* shift) {
  int pad = (xb / 2 + 1) * 2;
  std::vector<float> pr((size_t)pad * yb, 0.0f), pi((size_t)pad * yb, 0.0f),
      ps((size_t)pad * yb, 0.0f);
  for (int y = 0; y < yb; ++y) {
    memcpy(&pr[(size_t)y * pad], ref + (size_t)y * xb, xb * 4);
    memcpy(&pi[(size_t)y * pad], img + (size_t)y * xb, xb * 4);
  }
  auto normalize = [&](std::vector<float>& p) {
    float m = calc_moment(p.data(), xb, yb, pad, 1);
    float s = calc_moment(p.data(), xb, yb, pad, 2);
    s = s - m * m;
    if (s <= 0)
      s = 0.0f;
    else
      s = sqrtf(s);
    norm2d(p.data(), xb, yb, pad, m, s);
  };
  normalize(pr);
  // CalcCC::Stretch takes the stretch factor as a float (CalcCC.cu:318)
  double ds = cos(D2R * ref_tilt) / cos(D2R * tilt);
  float mat[3];
  stretch_matrix((float)ds, axis, mat);
  stretch(pi.data(), xb, yb, pad, mat, ps.data(), true);
  normalize(ps);
  round_edge(pr.data(), xb, yb, pad, xb * 0.5f, yb * 0.5f, xb * 1.0f, yb * 1.0f, 4);
  round_edge(ps.data(), xb, yb, pad, xb * 0.5f, yb * 0.5f, xb * 1.0f, yb * 1.0f, 4);
  auto R = fwd2d(pr.data(), xb, yb, pad, true);
  auto I = fwd2d(ps.data(), xb, yb, pad, true);
  std::vector<float> cc = xcorr_map(R, I, xb, yb, 400.0f);
  int w = xb, h = yb;
  int ssx = w * 8 / 20 * 2, ssy = h * 8 / 20 * 2;
  float pk = (float)-1e30;
  int px = 0, py = 0;
  int sx = (w - ssx) / 2, sy = (h - ssy) / 2;
  for (int y = sy; y < sy + ssy; ++y)
    for (int x = sx; x < sx + ssx; ++x) {
      if (pk >= cc[(size_t)y * w + x]) continue;
      px = x;
      py = y;
      pk = cc[(size_t)y * w + x];
    }
  if (px < 1)
    px = 1;
  else if (px > w - 2)
    px = w - 2;
  if (py < 1)
    py = 1;
  else if (py > h - 2)
    py = h - 2;
  size_t ic = (size_t)py * w + px;
  double a = (cc[ic + 1] + cc[ic - 1]) * 0.5f - cc[ic];
  double b = (cc[ic + 1] - cc[ic - 1]) * 0.5f;
  double c = (cc[ic + w] + cc[ic - w]) * 0.5f - cc[ic];
  double d = (cc[ic + w] - cc[ic - w]) * 0.5f;
  double dx = -b / (2 * a + 1e-30), dy = -d / (2 * c + 1e-30);
  if (fabs(dx) > 1) dx = 0;
  if (fabs(dy) > 1) dy = 0;
  shift[0] = (float)(px + dx) - w / 2;
  shift[1] = (float)(py + dy) - h / 2;
}

static void unstretch(oc_transform* t, int ref, int f, float* s) {
  double ds = cos(t->angles[ref] * D2R) / cos(t->angles[f] * D2R);
  float m[3];
  stretch_matrix(ds, t->param->rotate[f], m);
  float buf = s[0] * m[0] + s[1] * m[1];
  s[1] = s[0] * m[1] + s[1] * m[2];
  s[0] = buf;
}

float oc_transform_doit(oc_transform* t) {
  int nz = t->nz;
  size_t pix = (size_t)t->nx * t->ny, bpix = (size_t)t->xb * t->yb;
  std::vector<float> corr(nz * bpix);
  for (int i = 0; i < nz; ++i)
    correct_proj(t->stack + i * pix, t->nx, t->ny, t->param->shift_x[i], t->param->shift_y[i],
                 t->param->rotate[i], true, t->bin, true, false, corr.data() + i * bpix);
  float maxerr = 0.0f;
  float binx = t->nx * 1.0f / t->xb, biny = t->ny * 1.0f / t->yb;
  for (int z = 0; z < nz; ++z) {
    int r = find_ref_index(nz, t->angles.data(), z);
    if (r == z) continue;
    float sh[2];
    stretch_cc(corr.data() + r * bpix, corr.data() + z * bpix, t->xb, t->yb, t->angles[r],
               t->angles[z], t->param->rotate[z], sh);
    t->pshx[z] = sh[0] * binx;
    t->pshy[z] = sh[1] * biny;
    t->meas_x[z] = t->pshx[z];
    t->meas_y[z] = t->pshy[z];
    float e = (float)sqrt(t->pshx[z] * t->pshx[z] + t->pshy[z] * t->pshy[z]);
    if (e > maxerr) maxerr = e;
  }
  // UpdateShift (Transform.cpp:99-131)
  int zt = frame_idx_from_tilt(nz, t->angles.data(), 0.0f);
  for (int i = 0; i < nz; ++i) {
    // subtracts the live zero-tilt entry, which is itself zeroed at i == zt
    t->pshx[i] -= t->pshx[zt];
    t->pshy[i] -= t->pshy[zt];
  }
  float sum[2] = {0.0f, 0.0f};
  for (int i = zt - 1; i >= 0; --i) {
    sum[0] += t->pshx[i];
    sum[1] += t->pshy[i];
    unstretch(t, i + 1, i, sum);
    t->param->shift_x[i] += sum[0];
    t->param->shift_y[i] += sum[1];
  }
  sum[0] = sum[1] = 0.0f;
  for (int i = zt + 1; i < nz; ++i) {
    sum[0] += t->pshx[i];
    sum[1] += t->pshy[i];
    unstretch(t, i - 1, i, sum);
    t->param->shift_x[i] += sum[0];
    t->param->shift_y[i] += sum[1];
  }
  return maxerr;
}

// ---------------------------------------------------------------------------
// FindOffset.cu:85-238
float oc_find_offset(const float* stack, int nx, int ny, int nz, const float* angles,
                     oc_param* param) {
  const int bin = 4;
  int xb, yb;
  binned_size(nx, ny, bin, &xb, &yb);
  size_t pix = (size_t)nx * ny, bpix = (size_t)xb * yb;
  std::vector<float> corr(nz * bpix);
  for (int i = 0; i < nz; ++i)
    correct_proj(stack + i * pix, nx, ny, param->shift_x[i], param->shift_y[i], param->rotate[i],
                 false, bin, false, false, corr.data() + i * bpix);
  std::vector<float> a(angles, angles + nz);
  const int num = 31;
  std::vector<float> ccs(num);
  for (int n = 0; n < num; ++n) {
    float off = 0.0f + (n - num / 2) * 1.0f;
    for (int z = 0; z < nz; ++z) a[z] += off;
    int zt = frame_idx_from_tilt(nz, a.data(), 0.0f);
    int count = 0;
    float ccsum = 0.0f;
    for (int i = 0; i < nz; ++i) {
      if (i == zt) continue;
      int r = (i < zt) ? i + 1 : i - 1;
      double ds = cos(D2R * a[r]) / cos(D2R * a[i]);
      float m[3];
      stretch_matrix((float)ds, 0.0f, m);
      std::vector<float> st(bpix);
      stretch(corr.data() + i * bpix, xb, yb, xb, m, st.data(), false);
      const float* ref = corr.data() + r * bpix;
      double v[6] = {0, 0, 0, 0, 0, 0};
      for (size_t k = 0; k < bpix; ++k) {
        float v1 = ref[k];
        if (v1 < (float)-1e10) continue;
        float v2 = st[k];
        if (v2 < (float)-1e10) continue;
        v[0] += v1;
        v[1] += v2;
        v[2] += v1 * v1;
        v[3] += v2 * v2;
        v[4] += v1 * v2;
        v[5] += 1.0;
      }
      float f[6];
      for (int k = 0; k < 6; ++k) f[k] = (float)v[k];
      for (int k = 0; k < 5; ++k) f[k] /= f[5];
      // the reference subtracts the mean, not its square (FindOffset.cu:222-223)
      double s1 = f[2] - f[0], s2 = f[3] - f[1];
      double cc = f[4] - f[0] * f[1];
      if (s1 < 0) s1 = 0;
      if (s2 < 0) s2 = 0;
      s1 = sqrt(s1);
      s2 = sqrt(s2);
      cc = cc / (s1 * s2 + 1e-30);
      if (cc < -1)
        cc = -1;
      else if (cc > 1)
        cc = 1;
      ccsum += (float)cc;
      count++;
    }
    ccs[n] = ccsum / count;
    for (int z = 0; z < nz; ++z) a[z] -= off;
  }
  float maxcc = 0.0f, best = 0.0f;
  for (int n = 0; n < num; ++n) {
    float off = 0.0f + (n - num / 2) * 1.0f;
    if (ccs[n] > maxcc) {
      maxcc = ccs[n];
      best = off;
    }
  }
  param->angle_offset += best;
  return best;
}

// ---------------------------------------------------------------------------
// Process.cpp:329-372 (CorrectStack): rotate+shift, OutBin, random fill, no R-weight.
void oc_correct_stack(const float* stack, int nx, int ny, int nz, const oc_param* param,
                      int out_bin, float* out) {
  int xo, yo;
  binned_size(nx, ny, out_bin, &xo, &yo);
  size_t pix = (size_t)nx * ny, opix = (size_t)xo * yo;
  for (int i = 0; i < nz; ++i)
    correct_proj(stack + i * pix, nx, ny, param->shift_x[i], param->shift_y[i], param->rotate[i],
                 false, out_bin, true, false, out + i * opix);
}

// ---------------------------------------------------------------------------
// Process.cpp:34-92, 238-319
int oc_align(const float* raw, int nx, int ny, int nz, const float* file_angles, float offset,
             float pitch_angle, float zshift, int align_z, int out_bin, int nproj,
             oc_param* param, float* out, int verbose) {
  size_t pix = (size_t)nx * ny;
  std::vector<float> stack(pix * nz);
  oc_preprocess(raw, nx, ny, nz, file_angles, stack.data());
  std::vector<float> ang(file_angles, file_angles + nz);
  if (nz > 1 && ang[0] > ang[1]) std::reverse(ang.begin(), ang.end());
  for (int i = 0; i < nz; ++i) {
    param->shift_x[i] = 0.0f;
    param->shift_y[i] = 0.0f;
    param->rotate[i] = 0.0f;
  }
  param->angle_offset = 0.0f;
  int passes = 0;
  if (align_z != 0) {
    // mCoarseAlign
    if (pitch_angle == 0) {
      oc_transform* t = oc_transform_create(stack.data(), nx, ny, nz, ang.data(), param);
      for (int i = 1; i <= 3; ++i) {
        float e = oc_transform_doit(t);
        float ax = oc_tilt_axis(stack.data(), nx, ny, nz, ang.data(), param, 180.0f / i, 100);
        if (verbose) printf("oracle coarse %d: maxerr %8.2f axis %.2f\n", i, e, ax);
      }
      oc_transform_destroy(t);
    } else {
      for (int i = 0; i < nz; ++i) param->rotate[i] = pitch_angle;
    }
    if (offset == 0) {
      float o = oc_find_offset(stack.data(), nx, ny, nz, ang.data(), param);
      if (verbose) printf("oracle offset %.2f\n", o);
    } else {
      param->angle_offset = offset;
    }
    for (int z = 0; z < nz; ++z) ang[z] += param->angle_offset;
    // mProjAlign
    for (int i = 0; i < nz; ++i) {
      param->shift_x[i] = 0.0f;
      param->shift_y[i] = 0.0f;
    }
    oc_projalign* pa =
        oc_projalign_create(stack.data(), nx, ny, nz, ang.data(), param, zshift, align_z, nproj);
    auto once = [&]() {
      float last = oc_projalign_doit(pa);
      passes++;
      if (verbose) printf("oracle fLastErr %8.2f z0 %8.2f\n", last, pa->z0);
      for (int i = 1; i < 10; ++i) {
        float e = oc_projalign_doit(pa);
        passes++;
        if (verbose) printf("oracle fErr %8.2f z0 %8.2f\n", e, pa->z0);
        if (e <= last) {
          if (e < 2.0f) break;
          last = e;
        }
      }
    };
    once();
    for (int i = 1; i <= 4; ++i) {
      float ax = oc_tilt_axis(stack.data(), nx, ny, nz, ang.data(), param, 20.0f / i, 100);
      if (verbose) printf("oracle axis %.2f\n", ax);
      if (i == 1) once();
    }
    once();
    oc_projalign_destroy(pa);
  }
  if (out) oc_correct_stack(stack.data(), nx, ny, nz, param, out_bin, out);
  return passes;
}

}  // extern "C"
