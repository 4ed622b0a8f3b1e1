/* markerfree.h — C ABI of the B200 projection-matching alignment library.
 *
 * The reference program (ratolon/Markerfree) has no library API: its boundary is
 * the command line and the files (MRC stack, .rawtlt, .txt/.xf), and inside it the
 * C++ classes PreProcess, Transform, CalcTIltAxis, FindOffset, ProjAlign and
 * CorrTomoStack, which all mutate one shared AlignParam.  This header exposes the
 * same units one-for-one over plain pointers and sizes, so that a host program
 * (the bundled command-line tool, a ctypes/cffi binding, or another aligner) can
 * drive the pipeline stage by stage or as a whole.
 *
 * Conventions
 *  - Every function returns MF_OK (0) or a negative mf_status; the message of the
 *    last failure on the calling thread is returned by mf_last_error().
 *  - Host arrays are owned by the caller.  Device memory is owned by the library
 *    (one mf_context per GPU, one stream per context).
 *  - Images are row-major float32, x fastest; stacks are z-major (nz, ny, nx).
 *  - Angles are degrees; shifts are in pixels of the un-binned input stack.
 *  - A context is not thread-safe; use one context per host thread.
 */
#ifndef MARKERFREE_H
#define MARKERFREE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MF_API __attribute__((visibility("default")))
#else
#define MF_API
#endif

typedef enum {
  MF_OK = 0,
  MF_ERR_ARG = -1,       /* invalid argument (size, null pointer, range) */
  MF_ERR_CUDA = -2,      /* CUDA runtime error */
  MF_ERR_CUFFT = -3,     /* cuFFT error */
  MF_ERR_IO = -4,        /* file cannot be opened, read or written */
  MF_ERR_FORMAT = -5,    /* unsupported MRC mode / malformed file */
  MF_ERR_STATE = -6,     /* call out of order (e.g. DoIt before setup) */
  MF_ERR_NOMEM = -7,     /* device or host allocation failed / budget exceeded */
  MF_ERR_GEOMETRY = -8   /* no neighbouring tilt within range of a held-out tilt */
} mf_status;

/* AlignParam (Markerfree/src/method/Util.h:14-21): per-tilt shift and tilt-axis
 * angle plus the global tilt-angle offset.  Arrays hold nz entries each. */
typedef struct {
  float* shift_x;
  float* shift_y;
  float* rotate;
  float angle_offset;
} mf_align_param;

/* Command-line options that reach the alignment (Markerfree/src/main/opts.h:16-41,
 * -g O,P,Z,T,A,B,G / -p / -s).  `thickness` (T) is parsed but unused, as in the
 * reference. */
typedef struct {
  float offset;      /* O: tilt-angle offset; 0 = search it (FindOffset)        */
  float pitch_angle; /* P: tilt-axis angle; 0 = search it (Transform+axis)      */
  float zshift;      /* Z: initial rotation-centre z                            */
  int thickness;     /* T: unused                                               */
  int align_z;       /* A: slab thickness for projection matching; 0 = no align */
  int out_bin;       /* B: binning of the output stack                          */
  int gpu;           /* G: CUDA device ordinal                                  */
  int nproj;         /* -p: neighbours back-projected per held-out tilt         */
  int save_mode;     /* -s: 0 = .txt, 1 = .xf                                   */
  int precision;     /* mf_precision of the re-projection operands (not in the
                        reference; 0 = FP32, which is the reference's arithmetic) */
} mf_options;

/* Precision of the re-projection operands (the corrected stack rows and the
 * back-projection operator).  Accumulation is always FP32; peak fitting, shift
 * accumulation and the rotation-centre normal equation are FP64.  FP16/BF16 run
 * the re-projection on the tensor cores; 128-row tiles whose neighbour rows hold
 * a -1e30 sentinel (or, for FP16, a value beyond its range) are recomputed with
 * the exact FP32 gather. */
typedef enum { MF_PREC_FP32 = 0, MF_PREC_BF16 = 1, MF_PREC_FP16 = 2 } mf_precision;

typedef struct mf_context mf_context;
typedef struct mf_series mf_series;

/* ---- errors ------------------------------------------------------------- */
MF_API const char* mf_last_error(void);
MF_API const char* mf_version(void);
/* Test hook: device allocations number first .. first+count-1, counted in this
 * process from this call on, fail as if the device were full (MF_ERR_NOMEM)
 * without reaching the driver.  count 0 turns it off. */
MF_API void mf_debug_fail_device_allocations(int64_t first, int64_t count);

/* ---- context (replaces main.cpp:26 cudaSetDevice and the per-class plans) - */
MF_API int mf_context_create(int gpu, mf_context** out);
MF_API void mf_context_destroy(mf_context* ctx);
/* Blocks until all work queued on the context's stream has finished. */
MF_API int mf_context_sync(mf_context* ctx);
/* Count of library kernel launches issued on this context so far (graph
 * launches count every kernel node once per replay). */
MF_API int64_t mf_context_kernel_launches(mf_context* ctx);

/* ---- series: device-resident pre-processed stack --------------------------
 * Replaces Process::ReadStack + PreProcess::SetPositive/MassNormalization
 * (Markerfree/src/main/Process.cpp:129-236, Markerfree/src/method/Preprocess.cu:103-177):
 * the raw stack (file order) is reordered to ascending angles, made positive and
 * mass-normalised on the GPU and kept in HBM in place of the scratch buf.mrc. */
MF_API int mf_series_create(mf_context* ctx, const float* raw_stack, int nx, int ny, int nz,
                            const float* file_angles, mf_series** out);
/* Same, from a device buffer already holding the raw stack (file order). */
MF_API int mf_series_create_device(mf_context* ctx, const float* d_raw_stack, int nx, int ny,
                                   int nz, const float* file_angles, mf_series** out);
/* A stack that PreProcess has already treated (Markerfree/src/method/Preprocess.cu:
 * 103-177, the contents of the reference's buf.mrc that Process::mCoarseAlign and
 * mProjAlign read, Process.cpp:161-236): ascending angle order, made positive and
 * mass-normalised.  It is uploaded as it is, with `angles` in the same (ascending)
 * order; no pre-processing runs, so a caller that has run the reference's own
 * pre-processing hands over exactly the stack its later stages would read. */
MF_API int mf_series_create_preprocessed(mf_context* ctx, const float* stack, int nx, int ny,
                                         int nz, const float* angles, mf_series** out);
/* Destroy every series of a context before the context itself. */
MF_API void mf_series_destroy(mf_series* s);
/* Takes effect at the next mf_projalign_setup (a set-up pass of another
 * precision is discarded; mf_proj_align sets up by itself). */
MF_API int mf_series_set_precision(mf_series* s, mf_precision p);
/* Copies the pre-processed stack (nz*ny*nx floats) to host memory. */
MF_API int mf_series_get_stack(mf_series* s, float* host_out);
/* Angles used by the alignment stages (ascending, offset applied by the caller). */
MF_API int mf_series_set_angles(mf_series* s, const float* angles);
MF_API int mf_series_get_angles(mf_series* s, float* angles_out);
MF_API int mf_series_set_param(mf_series* s, const mf_align_param* p);
MF_API int mf_series_get_param(mf_series* s, mf_align_param* p);

/* ---- stages --------------------------------------------------------------- */
/* Transform::Setup + DoIt (Markerfree/src/method/Transform.cpp:24-157): stretch
 * cross-correlation of every tilt against its neighbour nearer zero tilt, shifts
 * accumulated outward.  The series keeps the Transform state between calls. */
MF_API int mf_transform_doit(mf_series* s, float* max_err);
/* CalcTIltAxis::DoIt (Markerfree/src/method/Rotate.cu:292-337): common-line search
 * over `num` candidate axes spanning `range` degrees; sets rotate[] for all tilts. */
MF_API int mf_tilt_axis(mf_series* s, float range, int num, float* axis_out);
/* mf_tilt_axis that also returns the score of each of the `num` candidates (the
 * common-line scores CalcTIltAxis::findTiltAxis ranks, Rotate.cu:468-528). */
MF_API int mf_tilt_axis_scores(mf_series* s, float range, int num, float* axis_out,
                               float* scores);
/* FindOffset::DoIt (Markerfree/src/method/FindOffset.cu:85-96): adds the best of
 * 31 one-degree tilt-angle offsets to param.angle_offset. */
MF_API int mf_find_offset(mf_series* s, float* offset_out);
/* ProjAlign::Setup (Markerfree/src/method/ProjAlign.cpp:48-125). */
MF_API int mf_projalign_setup(mf_series* s, float zshift, int align_z, int nproj);
/* ProjAlign::DoIt (Markerfree/src/method/ProjAlign.cpp:127-179): one projection-
 * matching pass over all tilts; returns the largest measured shift (px). */
MF_API int mf_projalign_doit(mf_series* s, float* max_err);
/* Rotation-centre z of the last pass (ProjAlign.cpp:459-486). */
MF_API int mf_projalign_z0(mf_series* s, float* z0);
/* Shifts measured in the last pass, xy[2*z], xy[2*z+1] for tilt z: un-binned px
 * before the rotation by the tilt axis, the values ProjAlign.cpp:203 prints
 * (zero for the zero tilt and for tilts not yet measured). */
MF_API int mf_projalign_measured(mf_series* s, float* xy);
/* Process::mCoarseAlign (Markerfree/src/main/Process.cpp:238-270); applies the
 * offset to the series' angles as the reference does. */
MF_API int mf_coarse_align(mf_series* s, float pitch_angle, float offset);
/* Process::mProjAlign + ProjAlignOnce (Process.cpp:272-319). */
MF_API int mf_proj_align(mf_series* s, float zshift, int align_z, int nproj, int* passes);
/* Process::CorrectStack (Process.cpp:329-372): rotate, shift and bin every tilt;
 * writes nz * (ny/out_bin/2*2) * (nx/out_bin/2*2) floats to host_out. */
MF_API int mf_correct_stack(mf_series* s, int out_bin, float* host_out);
/* Size of the output stack of mf_correct_stack. */
MF_API void mf_binned_size(int nx, int ny, int bin, int* xb, int* yb);

/* Process::DoIt minus file I/O (Process.cpp:34-92): pre-process, coarse-align,
 * projection-match and write the aligned stack (if aligned_out != NULL).
 * param arrays must hold nz entries; `passes` (optional) gets the DoIt count. */
MF_API int mf_align(mf_context* ctx, const float* raw_stack, int nx, int ny, int nz,
                    const float* file_angles, const mf_options* opt, mf_align_param* param,
                    float* aligned_out, int* passes);

/* Same as mf_align with the raw stack and the aligned output in device memory
 * (caller-owned, on the context's GPU); parameters are returned to the host. */
MF_API int mf_align_device(mf_context* ctx, const float* d_raw_stack, int nx, int ny, int nz,
                           const float* file_angles, const mf_options* opt, mf_align_param* param,
                           float* d_aligned_out, int* passes);
/* Process::DoIt (Markerfree/src/main/Process.cpp:34-92) from file to file, minus
 * the parameter file (write it with mf_save_param): reads the MRC stack (modes
 * 0/1/2) at in_mrc, aligns it with the angles as read from the .rawtlt file
 * (nz of them, nz from mf_mrc_info) and writes the aligned float32 stack to
 * out_mrc (NULL: no stack) with mf_mrc_write's header.  Slices stream through
 * two page-locked buffers in blocks of about 64 MB: a block is read from the
 * file while the previous one is copied to the GPU (8- and 16-bit samples are
 * converted to float there), and on output a block is written while the next is
 * copied back.  Results equal mf_align's on the same data. */
MF_API int mf_align_file(mf_context* ctx, const char* in_mrc, const float* file_angles,
                         const mf_options* opt, mf_align_param* param, const char* out_mrc,
                         int* passes);

/* Stage timing: when enabled, every projection-matching pass records CUDA events
 * around each held-out tilt's re-projection and cross-correlation work (also
 * inside the captured graph).  mf_context_stage_times returns, accumulated since
 * the last call and then reset: [0] re-projection ms, [1] re-projection
 * launches (one per held-out tilt), [2] cross-correlation + re-correction ms,
 * [3] passes, [4] re-projection algorithmic bytes (neighbour rows read, output
 * written, banded operator read), [5] re-projection multiply-adds. */
MF_API int mf_context_set_profiling(mf_context* ctx, int on);
MF_API int mf_context_stage_times(mf_context* ctx, double* out6);
/* Wall time per stage of the alignments run while stage timing was on (CUDA
 * events on the context's stream; each stage waits for its work), accumulated
 * since the last call and then reset, in ms: [0] series creation (upload,
 * pre-processing), [1] coarse alignment (stretch correlations, offset search),
 * [2] tilt-axis searches, [3] projection-matching set-up, [4] projection-matching
 * passes, [5] aligned-stack output; and the tilt-axis Radon kernel alone:
 * [6] its ms, [7] its launches, [8] the line samples it took, [9] its compulsory
 * bytes (each tilt image read once, the line values written once). */
MF_API int mf_context_stage_breakdown(mf_context* ctx, double* out10);
/* Diagnostic: CUDA's cosf and sinf of each of n float arguments (host arrays),
 * the values the kernels use where the reference's device code calls them.  A
 * CPU model of the path needs them to take the same nearest-neighbour decisions,
 * since they may differ from the correctly rounded values in the last place. */
MF_API int mf_device_cos_sin(mf_context* ctx, const float* x, int n, float* c, float* s);
/* The context's CUDA stream (cudaStream_t), for callers that order their own
 * work or timing events after the library's. */
MF_API void* mf_context_stream(mf_context* ctx);
/* Image rows per tensor-core tile of the FP16/BF16 re-projection (64, 128 or
 * 256; 0 = automatic: groups time each candidate on their first step and keep
 * the fastest per shape, single series choose from the image shape and the SM
 * count).  Read when a pass or a group is set up or a single re-projection is
 * queued. */
MF_API int mf_context_set_tc_rows(mf_context* ctx, int rows);
/* The tile-row choices the autotuner made in this context: up to max_rows rows
 * of 8 doubles each, {xb, yb, series per launch, precision, chosen rows, median
 * ms per launch with 256, 128 and 64 rows}; *n receives the number of rows
 * recorded (which may exceed max_rows). */
MF_API int mf_context_tc_tuning(mf_context* ctx, double* out, int max_rows, int* n);

/* ---- groups: many series in lockstep ---------------------------------------
 * Not in the reference, which aligns one series per process.  A group runs the
 * projection-matching pass (ProjAlign::DoIt, Markerfree/src/method/ProjAlign.cpp:
 * 127-179) of up to 32 series of one context and precision together: each stage
 * of the pass is one launch over all of them.  The series may differ in image
 * size, tilt count and binning; a series with fewer tilts has no work in the last
 * steps of a pass.  Per-series results equal those of aligning each series alone.
 * Destroy a group before its series. */
typedef struct mf_group mf_group;
/* ProjAlign::Setup for every series (their current angles and parameters). */
MF_API int mf_group_create(mf_series* const* series, int n, float zshift, int align_z, int nproj,
                           mf_group** out);
MF_API void mf_group_destroy(mf_group* g);
/* One pass over the series with active[i] != 0; max_err[i] gets the largest
 * measured shift of each active series (the reference's DoIt return value). */
MF_API int mf_group_doit(mf_group* g, const int* active, float* max_err);
/* Process::mProjAlign + ProjAlignOnce (Markerfree/src/main/Process.cpp:272-319) for
 * every series: shifts reset, then the reference's schedule with each series'
 * own break rule; passes[i] (optional) gets each series' pass count. */
MF_API int mf_group_proj_align(mf_group* g, int* passes);
/* Rotation-centre z of every series after the last pass. */
MF_API int mf_group_z0(mf_group* g, float* z0);
/* mf_align_device for n series of one shape (raw stacks and outputs in device
 * memory): coarse alignment per series, projection matching in groups.
 * params[i] must hold nz-entry arrays; d_out may be NULL (no output stack). */
MF_API int mf_align_many_device(mf_context* ctx, int n, const float* const* d_raw, int nx, int ny,
                                int nz, const float* const* file_angles, const mf_options* opt,
                                mf_align_param* params, float* const* d_out, int* passes);
/* One series of a batch: raw stack (file order) and aligned output in device
 * memory, its size, its angles as read (host), its slab thickness. */
typedef struct {
  const float* d_raw;        /* nz x ny x nx floats */
  int nx, ny, nz;
  const float* file_angles;  /* nz angles, host memory */
  int align_z;               /* -g A of this series; 0 = the options' align_z */
  float* d_out;              /* aligned stack (nz x ny/out_bin x nx/out_bin), or NULL */
} mf_series_desc;
/* Process::DoIt minus file I/O (Markerfree/src/main/Process.cpp:34-92) for n
 * series of any sizes, tilt counts and slab thicknesses: each series is
 * pre-processed, coarse-aligned stage by stage with the others of its group of up
 * to 32, projection-matched with them in one lockstep group, and corrected into
 * its d_out.  params[i] must hold nz_i-entry arrays; passes (optional) gets each
 * series' pass count. */
MF_API int mf_align_batch_device(mf_context* ctx, int n, const mf_series_desc* series,
                                 const mf_options* opt, mf_align_param* params, int* passes);

/* ---- serving: continuous batching of requests ------------------------------
 * Not in the reference.  A server keeps `workers` streams busy with requests
 * (tilt series) that arrive at any time: a request is admitted when its
 * estimated device memory fits in `hbm_budget` bytes (0 = 65% of the free
 * memory), prepared on its own (upload, pre-processing, coarse alignment), then
 * projection-matched in a group with other prepared requests of any shape that
 * share its precision, -p and z shift (up to `max_group`).  A worker runs a full
 * group first, then prepares admitted requests (so that more requests join the
 * ready groups), then runs a group
 * whose oldest request has waited `group_wait_ms` or has no companion on the way;
 * no request waits longer than 20 x `group_wait_ms` once prepared.  A request's
 * result equals the one it gets when aligned alone. */
typedef struct mf_server mf_server;
MF_API int mf_server_create(int gpu, size_t hbm_budget, int max_group, int workers,
                            double group_wait_ms, mf_server** out);
/* Queue a request.  raw (nz x ny x nx, file order) and aligned_out (optional,
 * the mf_correct_stack layout) are caller-owned host memory that must stay valid
 * until mf_server_wait has returned for the job. */
MF_API int mf_server_submit(mf_server* s, const float* raw, int nx, int ny, int nz,
                            const float* file_angles, const mf_options* opt, float* aligned_out,
                            int64_t* job_id);
/* Block until the job is done (or timeout_s passes: MF_ERR_STATE).  param arrays
 * (nz entries), passes and latency_s (submit to done) are optional. */
MF_API int mf_server_wait(mf_server* s, int64_t job_id, double timeout_s, mf_align_param* param,
                          int* passes, double* latency_s);
/* out8: [0] jobs done, [1] series/min from the first submit to the last
 * completion, [2] p50 and [3] p99 latency (s), [4] peak admitted bytes, [5]
 * groups run, [6] mean group size, [7] seconds from first submit to last done. */
MF_API int mf_server_stats(mf_server* s, double* out8);
/* The memory budget: as created (budget0), as learned (budget_now: lowered to
 * what the other requests held whenever a prepare or a group set-up found the
 * device full while others held memory -- such a request is retried, not
 * failed), and how many such retries there were.  Any output may be null. */
MF_API int mf_server_memory(mf_server* s, size_t* budget0, size_t* budget_now, int64_t* retries);
/* Finishes every submitted request, then releases the workers. */
MF_API void mf_server_destroy(mf_server* s);

/* ---- single kernels on caller-owned device memory (same stream semantics:
 * the call is ordered on the context stream and returns after queuing). ------ */
/* CorrTomoStack::mCorrectProj (Markerfree/src/method/CorrStack.cu:370-397) for one
 * projection: d_proj (ny x nx) -> d_out (ny/bin/2*2 x nx/bin/2*2). */
MF_API int mf_dev_correct_proj(mf_context* ctx, const float* d_proj, int nx, int ny,
                               float shift_x, float shift_y, float tilt_axis, int only_shift,
                               int bin, int random_fill, int rweight, float* d_out);
/* CalcReprojFBP::FindProjRange (Markerfree/src/method/CalcReproj.cu:206-259). */
MF_API int mf_find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                              int nproj, int* range2);
/* CalcReprojFBP::DoIt (CalcReproj.cu:180-311): back-project tilts [istart, iend] of
 * the corrected stack d_corr (nz x yb x xb) into a 2*xb x thickness slab per row
 * and re-project it at angles[iproj] into d_out (yb x xb).  method 0 = exact
 * per-sample gather, 1 = banded operator in FP32 (the FP32 production path),
 * 2 / 3 = the same operator applied on the tensor cores with FP16 / BF16 operands
 * and FP32 accumulation (the mixed-precision production path). */
MF_API int mf_dev_reproject(mf_context* ctx, const float* d_corr, int xb, int yb, int nz,
                            const float* angles, int iproj, int istart, int iend, int thickness,
                            int method, float* d_out);
/* The exact re-projection of mf_dev_reproject (method 0) for callers that cannot
 * allocate device memory.  It has no counterpart in the reference.  Hosts such as
 * acquisition programs that reserve the GPU's memory for their own buffers, or
 * real-time loops in which a cudaMalloc/cudaFree could synchronise the device,
 * cannot let the library grow scratch buffers; this entry point allocates
 * nothing.  Its per-neighbour table lives in a static device array of at most
 * 256 neighbour tilts (3 KB, held by every GPU that loads the library until the
 * process exits); more neighbours are rejected with MF_ERR_ARG.  The first call
 * on a device looks the array's address up, so make that first call before any
 * stream capture on the device.  All calls share the array: calls whose kernels
 * overlap on the GPU (e.g. on two streams) race.  `stream` is a cudaStream_t
 * (NULL = the legacy default stream) of the current device; the call returns
 * after queuing the work. */
MF_API int mf_dev_reproject_noalloc(void* stream, const float* d_corr, int xb, int yb, int nz,
                                    const float* angles, int iproj, int istart, int iend,
                                    int thickness, float* d_out);
/* ProjAlign::MeaAlignProj + PAFindPeak (ProjAlign.cpp:243-375): shift (binned px)
 * of d_proj against d_reproj, both yb x xb. */
MF_API int mf_dev_measure_shift(mf_context* ctx, const float* d_reproj, const float* d_proj,
                                int xb, int yb, float* shift2, float* peak);

/* ---- files (MrcStackM, Process::ReadAngles, SaveParam) ---------------------- */
/* MRC header fields (Markerfree/src/mrc/mrcheader.h:24-96); modes 0, 1, 2 read. */
MF_API int mf_mrc_info(const char* path, int* nx, int* ny, int* nz, int* mode);
MF_API int mf_mrc_read(const char* path, float* out);
/* Float32 MRC with the reference's header (InitializeHeader + UpdateHeader:
 * statistics of the middle slice only, mrcstack.cpp:421-501). */
MF_API int mf_mrc_write(const char* path, const float* data, int nx, int ny, int nz);
/* Whitespace-separated floats (Process.cpp:186-206); *n gets the count read. */
MF_API int mf_read_angles(const char* path, float* out, int max, int* n);
/* Process::CollectParam + SaveParam::GetParam(bin=1, mode, inv)
 * (Markerfree/src/main/Process.cpp:399-418, Markerfree/src/method/SaveParam.cpp:122-183):
 * writes <out>.txt (mode 0) or <out>.xf (mode 1), ".mrc" in the output path
 * replaced; file_angles are the angles in file order (reversed here when they
 * descend, which also reverses the .xf rows). */
MF_API int mf_save_param(const char* output_path, int mode, const mf_align_param* p,
                         const float* file_angles, int nz, int raw_nx, int raw_ny, int out_bin,
                         float elapsed_s);

#ifdef __cplusplus
}
#endif
#endif /* MARKERFREE_H */
