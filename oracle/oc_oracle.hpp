// CPU oracle for the Markerfree projection-matching alignment path.
//
// TEST INFRASTRUCTURE ONLY.  This is a single-threaded-per-item FP32 restatement
// of the reference algorithm (FFTs in FP64) used by tests/, by the smoke check and
// by bench.py's CPU-baseline leg.  The product path (markerfree_b200) never links,
// loads or calls it.
//
// Every function cites the reference file:line it restates.  Paths are relative to
// the reference project root (Markerfree/src/...).
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

// Mirror of AlignParam (Markerfree/src/method/Util.h:14-21).
typedef struct {
  float* shift_x;
  float* shift_y;
  float* rotate;
  float angle_offset;
} oc_param;

// ---- helpers (Markerfree/src/method/Util.cpp:8-35) ----
int oc_frame_idx_from_tilt(int nz, const float* angles, float tilt);
int oc_find_ref_index(int nz, const float* angles, int z);

// ---- pre-processing (Markerfree/src/method/Preprocess.cu:103-250) ----
// raw: nz slices of nx*ny in file order; angles: as read from the .rawtlt file.
// out: angle-ascending, positive, mass-normalised float stack.
void oc_preprocess(const float* raw, int nx, int ny, int nz, const float* angles, float* out);

// ---- stack correction (Markerfree/src/method/CorrStack.cu) ----
void oc_binned_size(int nx, int ny, int bin, int* xb, int* yb);
// One projection: rotate by tilt_axis (deg, ignored when only_shift), shift,
// nearest-neighbour resample with optional random fill, bin, optional R-weight.
void oc_correct_proj(const float* proj, int nx, int ny, float shift_x, float shift_y,
                     float tilt_axis_deg, int only_shift, int bin, int random_fill,
                     int rweight, float* out);

// ---- re-projection (Markerfree/src/method/CalcReproj.cu) ----
void oc_find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                        int nproj, int* range2);
// Back-project neighbours [istart, iend] of the corrected stack (nz x yb x xb)
// into a W=2*xb by T slab per row and re-project it at angles[iproj].
void oc_reproject(const float* corr, int xb, int yb, int nz, const float* angles, int iproj,
                  int istart, int iend, int thickness, float* out);

// ---- CC measurement (Markerfree/src/method/ProjAlign.cpp:243-375) ----
// Returns the shift (binned px) of proj against reproj; peak value in *peak.
void oc_measure_shift(const float* reproj, const float* proj, int xb, int yb, float* shift2,
                      float* peak);

// ---- projection-matching state machine (ProjAlign.cpp, Process.cpp:272-319) ----
typedef struct oc_projalign oc_projalign;
oc_projalign* oc_projalign_create(const float* stack, int nx, int ny, int nz, const float* angles,
                                  oc_param* param, float zshift, int align_z, int nproj);
float oc_projalign_doit(oc_projalign* pa);
float oc_projalign_z0(const oc_projalign* pa);
// Per tilt (x, y) shift measured by the last pass, un-binned px, before the
// tilt-axis rotation (the values the reference prints per held-out tilt).
void oc_projalign_measured(const oc_projalign* pa, float* xy);
int oc_projalign_bin(const oc_projalign* pa);
void oc_projalign_destroy(oc_projalign* pa);

// ---- tilt axis (Markerfree/src/method/Rotate.cu:292-572) ----
float oc_tilt_axis(const float* stack, int nx, int ny, int nz, const float* angles,
                   oc_param* param, float range, int num);
// Same, also returning the `num` candidate scores.
float oc_tilt_axis_scores(const float* stack, int nx, int ny, int nz, const float* angles,
                          oc_param* param, float range, int num, float* scores_out);

// ---- coarse alignment (Transform.cpp, FindOffset.cu) ----
typedef struct oc_transform oc_transform;
oc_transform* oc_transform_create(const float* stack, int nx, int ny, int nz, const float* angles,
                                  oc_param* param);
float oc_transform_doit(oc_transform* t);
void oc_transform_measured(const oc_transform* t, float* x, float* y);
void oc_transform_destroy(oc_transform* t);
float oc_find_offset(const float* stack, int nx, int ny, int nz, const float* angles,
                     oc_param* param);

// ---- output (Process.cpp:329-372) ----
void oc_correct_stack(const float* stack, int nx, int ny, int nz, const oc_param* param,
                      int out_bin, float* out);

// ---- whole pipeline (Process.cpp:34-92) minus file I/O ----
// raw stack in file order and the file's angles; fills param (nz entries) and
// the aligned stack (if out != NULL).  Returns the number of DoIt passes run.
int oc_align(const float* raw, int nx, int ny, int nz, const float* file_angles, float offset,
             float pitch_angle, float zshift, int align_z, int out_bin, int nproj,
             oc_param* param, float* out, int verbose);

#ifdef __cplusplus
}
#endif
