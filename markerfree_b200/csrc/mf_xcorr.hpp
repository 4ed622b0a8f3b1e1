// Launch wrappers of mf_xcorr.cu, mf_correct.cu (pre-processing), mf_axis.cu
// and mf_offset.cu.
#pragma once
#include "mf_internal.hpp"

namespace mf {

// Masked mean (and std) of each image, then normalise + round-edge mask into the
// padded FFT layout.  Image i is read from src + i*src_img_stride, except image 1
// which is read from src1 when src1 is not null.  d_part needs
// moment_parts(h) * nimg entries.
// mask: the w x h table of make_round_mask for the same geometry, or null
int norm_mask_pad(Context* c, const float* src, const float* src1, int src_stride,
                  size_t src_img_stride, int w, int h, int pad, size_t dst_img_stride, int nimg,
                  int with_std, float cx, float cy, float msx, float msy, float power,
                  const float* mask, float* dst, double2* d_part, float2* d_stats,
                  cudaStream_t st);
// GRoundEdge factors of a w x h image (-1 where the mask is zero)
int make_round_mask(Context* c, int w, int h, float cx, float cy, float msx, float msy,
                    float power, float* d_mask, cudaStream_t st);
int moment_parts(int h);
// Group forms (one launch over the series of a group at one step; each series
// with its own geometry and buffers, see GroupSeriesDev): PANorm of the pair
// (re-projection, held-out tilt) into the series' cc buffer; the conjugate
// product and filter of the pair's spectra; the peak + parameter update;
// FitRotCenterZ; the pass maximum.
int norm_mask_pad_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                        const int* active, int nseries, int xb_max, int yb_max, int pad_max,
                        cudaStream_t st);
int xcorr_filter_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                       const int* active, int nseries, int cmp_max, int yb_max, float bfactor,
                       cudaStream_t st);
int pa_peak_update_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                         const int* active, int nseries, cudaStream_t st);
int fit_z0_group(Context* c, const GroupSeriesDev* ser, const int* active, int nseries,
                 cudaStream_t st);
int max_err_group(Context* c, const GroupSeriesDev* ser, const int* active, int nseries,
                  float* d_out, cudaStream_t st);

int xcorr_filter(Context* c, const cufftComplex* ref, size_t ref_stride, const int* d_ref_idx,
                 cufftComplex* img, size_t img_stride, int npairs, int cmp, int ny, float bfactor,
                 float scale, cudaStream_t st);
// d_sx64/d_sy64 (FP16/BF16 modes; null in FP32 mode): FP64 accumulators of the
// shifts, of which d_sx/d_sy receive the float values.
int pa_peak_update(Context* c, const float* map, int stride, int xb, int yb, float2* d_part,
                   int ip, int nx, int ny, const float* d_angles, float* d_sx, float* d_sy,
                   double* d_sx64, double* d_sy64, const float* d_rot, const float* d_z0,
                   float* d_err, float* d_meas, cudaStream_t st);
int pa_peak_only(Context* c, const float* map, int stride, int xb, int yb, float2* d_part,
                 float* d_out, cudaStream_t st);
int cc_peaks(Context* c, const float* maps, size_t map_stride, int stride, int w, int h, int nmaps,
             float2* d_part, float2* d_shifts, cudaStream_t st);
constexpr int kPeakParts = 256;  // partial blocks of the single-map peak search
int fit_z0(Context* c, int nz, int zt, const float* d_angles, float* d_sx, float* d_sy,
           double* d_sx64, double* d_sy64, const float* d_rot, float* d_z0, cudaStream_t st);
int max_err(Context* c, const float* d_err, const int* d_order, int n, float* d_out,
            cudaStream_t st);
int stretch_many(Context* c, const float* src, size_t src_img_stride, const int* d_src_idx,
                 int gw, int h, int stride, const float* d_mats, int n, int randfill, float* dst,
                 size_t dst_img_stride, cudaStream_t st);
void stretch_matrix(float dstretch, float tilt_axis, float* m);

int preprocess_device(Context* c, float* d_stack, int nx, int ny, int nz,
                      const float* file_angles, cudaStream_t st);

// Common-line tilt-axis search over all tilts (Rotate.cu), queued without a host
// wait: tilt_axis_scores_enqueue launches every kernel of one search and copies the
// candidates' scores into a page-locked slot of the context; once the stream has
// been synchronised, tilt_axis_scores_finish returns them (num floats) and books
// the Radon kernel's stage timing.  The caller applies the arg-max rule.
struct AxisJob {
  float* h_scores = nullptr;              // page-locked, num floats
  unsigned long long* h_count = nullptr;  // page-locked, samples taken (stage timing)
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int num = 0, L = 0, nx = 0, ny = 0, nz = 0;
  AxisJob() = default;
  AxisJob(const AxisJob&) = delete;
  AxisJob& operator=(const AxisJob&) = delete;
  ~AxisJob();
};
// stack_t: the same stack column-major per tilt (transpose_stack); d_neg[z]: image
// z holds a value below zero (null: assume it may); slot: the context's pinned
// slot the scores go to (unique among the searches queued before one wait).
int tilt_axis_scores_enqueue(Context* c, cufftHandle plan, const float* stack,
                             const float* stack_t, const int* d_neg, int nx, int ny, int nz,
                             const float* angles, const float* sx, const float* sy, int zt,
                             const float* rot_cand, int num, int line_len, int slot, AxisJob* job,
                             cudaStream_t st);
int tilt_axis_scores_finish(Context* c, AxisJob* job, std::vector<float>* scores);
// d_c[i] = cosf(d_x[i]), d_s[i] = sinf(d_x[i]) on the device.
int device_cos_sin(Context* ctx, const float* d_x, int n, float* d_c, float* d_s,
                   cudaStream_t st);
// out[z][x][y] = stack[z][y][x] for every tilt; neg[z] = 1 when image z holds a
// value below zero, else 0.
int transpose_stack(Context* c, const float* stack, int width, int height, int nz, float* out,
                    int* neg, cudaStream_t st);

// Tilt-angle offset search (FindOffset.cu): sums[6] per (offset, pair).
struct OffsetPair {
  int ref, img;
  float m0, m1, m2;
};
int offset_moments(Context* c, const float* corr, int w, int h, const OffsetPair* d_pairs,
                   int npairs, double* d_out, cudaStream_t st);

}  // namespace mf
