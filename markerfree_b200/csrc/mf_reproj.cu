// Re-projection of a held-out tilt from its back-projected neighbours.
//
// Reference: Markerfree/src/method/CalcReproj.cu.  For every image row y the
// reference back-projects the K neighbour rows into a 2*Xb x T slab
// (mGBackProj, :17-64, nearest-neighbour sinogram samples weighted by
// cos((theta_h - theta_i) * 0.01745) and cos(theta_i)), then sums each detector
// column's ray through the slab at the held-out angle (mGForProj, :68-124, mean of
// valid samples, -1e30 when fewer than 0.8 of the ray length are valid).  It
// launches both kernels once per row, Yb times per held-out tilt.
//
// Two implementations live here:
//  * an exact per-sample gather that evaluates the reference's arithmetic for all
//    rows in one launch (used for rows that contain -1e30 sentinels and as the
//    parity baseline);
//  * the production path.  Which slab cell a ray sample lands in, which sinogram
//    bin each neighbour contributes to that cell and with what weight depend only
//    on the angles, the slab thickness and the image width — never on the row or
//    on pixel values, as long as no neighbour value is a sentinel.  So for a held-
//    out tilt the whole back-project/re-project pair is one fixed linear map from
//    the K neighbour rows to the output row, the same for every row: a banded
//    matrix.  It is built once per series (the angles do not change while
//    projection matching runs) and applied to all Yb rows as a dense-tiled GEMM.
#include <atomic>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <cstdio>

#include "mf_internal.hpp"

namespace mf {

// ---------------------------------------------------------------------------
// Host geometry (CalcReproj.cu:43-44, 301-303).
void reproj_geometry(const float* angles, int ip, int i0, int i1, int xb, int yb, int thick,
                     ReprojGeom* g) {
  g->ip = ip;
  g->i0 = i0;
  g->i1 = i1;
  g->nk = i1 - i0 + 1;
  g->xb = xb;
  g->yb = yb;
  g->thick = thick;
  const float pa = angles[ip];
  g->bp.resize((size_t)g->nk * 3);
  for (int k = 0; k < g->nk; ++k) {
    float a = angles[i0 + k];
    g->bp[3 * k + 0] = cos_f((pa - a) * kBpD2R);
    float v = a * kBpD2R;
    g->bp[3 * k + 1] = cos_f(v);
    g->bp[3 * k + 2] = sin_f(v);
  }
  g->fcos = (float)std::cos(kD2R * pa);
  g->fsin = (float)std::sin(kD2R * pa);
  g->ray_len = (int)((float)thick / g->fcos + 0.5f);
}

// Back-projection weights and directions with CUDA's cosf/sinf, as mGBackProj
// evaluates them (CalcReproj.cu:43-46): per neighbour (w, cos, sin).
struct BpArgs {
  float pa;
  int nk;
  float a[kMaxBpNeighbours];
};
__global__ void k_bp_table(BpArgs args, float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= args.nk) return;
  const float a = args.a[k];
  out[3 * k + 0] = cosf(__fmul_rn(__fsub_rn(args.pa, a), kBpD2R));
  const float v = __fmul_rn(a, kBpD2R);
  out[3 * k + 1] = cosf(v);
  out[3 * k + 2] = sinf(v);
}

int bp_table_device(Context* c, const float* angles, int ip, int i0, int nk, float* d_out,
                    cudaStream_t st) {
  if (nk < 1 || nk > kMaxBpNeighbours)
    return set_error(MF_ERR_ARG, "%d neighbour tilts (1..%d supported)", nk, kMaxBpNeighbours);
  BpArgs args{};
  args.pa = angles[ip];
  args.nk = nk;
  for (int k = 0; k < nk; ++k) args.a[k] = angles[i0 + k];
  k_bp_table<<<(nk + 127) / 128, 128, 0, st>>>(args, d_out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int fill_bp_device(Context* c, const float* angles, std::vector<ReprojGeom>* geoms,
                   cudaStream_t st) {
  size_t total = 0;
  for (const ReprojGeom& g : *geoms) total += 3 * (size_t)g.nk;
  if (total == 0) return MF_OK;
  DevBuf d;
  MF_TRY(d.alloc(sizeof(float) * total));
  size_t off = 0;
  for (const ReprojGeom& g : *geoms) {
    MF_TRY(bp_table_device(c, angles, g.ip, g.i0, g.nk, d.as<float>() + off, st));
    off += 3 * (size_t)g.nk;
  }
  std::vector<float> h(total);
  MF_CHECK_CUDA(cudaMemcpyAsync(h.data(), d.p, sizeof(float) * total, cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  off = 0;
  for (ReprojGeom& g : *geoms) {
    g.bp.assign(h.begin() + off, h.begin() + off + 3 * (size_t)g.nk);
    off += 3 * (size_t)g.nk;
  }
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Device geometry helpers.  Every step is an explicitly rounded IEEE operation,
// and a multiply-add is fused exactly where nvcc fuses the reference's
// expressions (its default contraction: in a*b + c and c - a*b the product is
// fused; in a*b + c*d the first product): cell and bin indices then agree bit for
// bit with the reference binary and with a C evaluation that uses fmaf at the
// same places.
struct RayStart {
  float tx, tz, zst;
};

__device__ __forceinline__ RayStart ray_start(int bx, int xb, int W, int T, float fcos,
                                              float fsin, int L) {
  float fxp = __fsub_rn(__fadd_rn((float)bx, 0.5f), __fmul_rn((float)xb, 0.5f));
  RayStart r;
  r.tx = __fmaf_rn(fxp, fcos, __fmul_rn((float)W, 0.5f));
  r.tz = __fmaf_rn(fxp, fsin, __fmul_rn((float)T, 0.5f));
  r.zst = __fsub_rn(__fdiv_rn(__fmul_rn(-fxp, fsin), fcos), __fmul_rn(0.5f, (float)L));
  return r;
}

// Sample j of a ray; returns false when outside [0, W-1) x [0, T-1).
__device__ __forceinline__ bool ray_cell(const RayStart& r, int j, int W, int T, float fcos,
                                         float fsin, int* ix, int* iz) {
  float fz = __fadd_rn((float)j, r.zst);
  float X = __fmaf_rn(-fz, fsin, r.tx);
  float Z = __fmaf_rn(fz, fcos, r.tz);
  if (!(X >= 0.0f && X < (float)(W - 1) && Z >= 0.0f && Z < (float)(T - 1))) return false;
  *ix = (int)X;
  *iz = (int)Z;
  return true;
}

// Sinogram bin of neighbour (c, s) for slab cell (ix, iz); -1 when out of range.
__device__ __forceinline__ int cell_bin(int ix, int iz, int W, int T, float c, float s,
                                        float cent, int xb) {
  float fx = __fsub_rn(__fadd_rn((float)ix, 0.5f), __fmul_rn((float)W, 0.5f));
  float fz = __fsub_rn(__fadd_rn((float)iz, 0.5f), __fmul_rn((float)T, 0.5f));
  float v = __fadd_rn(__fmaf_rn(fx, c, __fmul_rn(fz, s)), cent);
  if (v < 0.0f || v > (float)(xb - 1)) return -1;
  return (int)v;
}

__device__ void exact_rows(const float* __restrict__ corr, int xb, size_t pix,
                           const float* __restrict__ bp, int i0, int nk, float fcos, float fsin,
                           int L, int T, int bx, int ya, int yz, float* __restrict__ out);

// ---------------------------------------------------------------------------
// Exact path: one thread per detector column; a block covers `rows_per_block`
// image rows.  With row flags (the fallback after the banded apply) a block
// handles one row tile and leaves at once when that tile holds no sentinel.
__global__ void k_reproject_exact(const float* __restrict__ corr, int xb, int yb, size_t pix,
                                  const float* __restrict__ bp, int i0, int nk, float fcos,
                                  float fsin, int L, int T, const int* __restrict__ rowflags,
                                  const int* __restrict__ tflags, int rows_per_block,
                                  float* __restrict__ out) {
  if (rowflags && rowflags[blockIdx.y] == 0) return;
  if (tflags) {
    // per-tilt flags of the 16-bit copy: recompute the tile if any neighbour's is set
    int any = 0;
    for (int k = 0; k < nk; ++k)
      for (int q = 0; q < kFlagParts; ++q)
        any |= tflags[((size_t)(i0 + k) * gridDim.y + blockIdx.y) * kFlagParts + q];
    if (!any) return;
  }
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= xb) return;
  const int ya = blockIdx.y * rows_per_block, yz = min(yb, ya + rows_per_block);
  exact_rows(corr, xb, pix, bp, i0, nk, fcos, fsin, L, T, bx, ya, yz, out);
}

// Rows [ya, yz) of column bx with the reference's per-sample arithmetic.
__device__ void exact_rows(const float* __restrict__ corr, int xb, size_t pix,
                           const float* __restrict__ bp, int i0, int nk, float fcos, float fsin,
                           int L, int T, int bx, int ya, int yz, float* __restrict__ out) {
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  const RayStart r = ray_start(bx, xb, W, T, fcos, fsin, L);
  for (int y = ya; y < yz; ++y) {
    float sum = 0.0f;
    int cnt = 0;
    for (int j = 0; j < L; ++j) {
      int ix, iz;
      if (!ray_cell(r, j, W, T, fcos, fsin, &ix, &iz)) continue;
      float fint = 0.0f, fcount = 0.0f;
      for (int k = 0; k < nk; ++k) {
        float w = bp[3 * k], c = bp[3 * k + 1], s = bp[3 * k + 2];
        int b = cell_bin(ix, iz, W, T, c, s, cent, xb);
        if (b < 0) continue;
        float v = corr[(size_t)(i0 + k) * pix + (size_t)y * xb + b];
        if (v < -1e10f) continue;  // mDIntProj turns it into -1e30, then skipped
        fint = __fmaf_rn(__fmul_rn(v, c), w, fint);
        fcount = __fadd_rn(fcount, w);
      }
      float cell = (fcount < 0.001f) ? kSentinel : __fdiv_rn(fint, fcount);
      if (cell >= -1e10f) {
        sum = __fadd_rn(sum, cell);
        cnt += 1;
      }
    }
    float res =
        ((float)cnt < __fmul_rn(0.8f, (float)L)) ? kSentinel : __fdiv_rn(sum, (float)cnt);
    out[(size_t)y * xb + bx] = res;
  }
}

int launch_reproject_exact(Context* c, const float* corr, int xb, int yb, size_t pix,
                           const float* d_bp, int i0, int nk, float fcos, float fsin, int ray_len,
                           int thick, const int* d_rowflags, float* out, cudaStream_t st) {
  const int rpb = d_rowflags ? kApplyTileY : 1;
  dim3 blk(128, 1), grd((xb + 127) / 128, (yb + rpb - 1) / rpb);
  k_reproject_exact<<<grd, blk, 0, st>>>(corr, xb, yb, pix, d_bp, i0, nk, fcos, fsin, ray_len,
                                         thick, d_rowflags, nullptr, rpb, out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Group form: blockIdx.z = series, with its own geometry.  A row tile is recomputed
// when its flags say so (any neighbour's 16-bit tile flag, or the FP32 apply's row
// flag of this step).
__global__ void k_reproject_exact_group(const GroupSeriesDev* __restrict__ ser,
                                        const GroupStepDev* __restrict__ steps,
                                        const int* __restrict__ active,
                                        const float* __restrict__ bps, int tc,
                                        const int* __restrict__ rowflags, int ytiles_max) {
  const int b = blockIdx.z;
  if (active && active[b] == 0) return;
  const GroupStepDev S = steps[b];
  if (S.ip < 0) return;
  const GroupSeriesDev& G = ser[b];
  const int yblk = blockIdx.y;
  if (yblk >= G.ytiles) return;
  if (tc) {
    int any = 0;
    for (int k = 0; k < S.nk; ++k)
      for (int q = 0; q < kFlagParts; ++q)
        any |= G.tflags[((size_t)(S.i0 + k) * G.ytiles + yblk) * kFlagParts + q];
    if (!any) return;
  } else if (rowflags[b * ytiles_max + yblk] == 0) {
    return;
  }
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= G.xb) return;
  const int ya = yblk * kApplyTileY, yz = min(G.yb, ya + kApplyTileY);
  exact_rows(G.corr, G.xb, G.bpix, bps + S.bp_off, S.i0, S.nk, S.fcos, S.fsin, S.ray_len,
             S.thick, bx, ya, yz, G.reproj);
}

int launch_reproject_exact_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                                 const int* active, int nseries, int xb_max, int ytiles_max,
                                 const float* d_bp, bool tc, const int* rowflags,
                                 cudaStream_t st) {
  dim3 blk(128, 1), grd((xb_max + 127) / 128, ytiles_max, nseries);
  k_reproject_exact_group<<<grd, blk, 0, st>>>(ser, steps, active, d_bp, tc ? 1 : 0, rowflags,
                                               ytiles_max);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

int launch_reproject_exact_flagged(Context* c, const float* corr, int xb, int yb, size_t pix,
                                   const float* d_bp, int i0, int nk, float fcos, float fsin,
                                   int ray_len, int thick, const int* tflags, float* out,
                                   cudaStream_t st) {
  dim3 blk(128, 1), grd((xb + 127) / 128, (yb + kApplyTileY - 1) / kApplyTileY);
  k_reproject_exact<<<grd, blk, 0, st>>>(corr, xb, yb, pix, d_bp, i0, nk, fcos, fsin, ray_len,
                                         thick, nullptr, tflags, kApplyTileY, out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Operator build for a set of held-out tilts (one launch per pass over all of
// them).  Pass 1: per column the number of valid ray samples and, per
// neighbour, the range of sinogram bins touched.
struct OpGeomDev {
  int nk, ray_len, T, bp_off;  // bp_off: float offset of (w, c, s) triples
  float fcos, fsin;
  int lohi_off;  // int offset of this tilt's lo/hi arrays (xb * nk each)
  int tile_off;  // first OpTile of this tilt
  int seg_off;   // first int2 of this tilt's segment table (ntiles * nk)
  int i0;        // absolute index of the first neighbour tilt
};

__global__ void k_op_scan(int xb, const OpGeomDev* __restrict__ geoms,
                          const float* __restrict__ bps, int* __restrict__ cnt,
                          int* __restrict__ lo, int* __restrict__ hi) {
  const OpGeomDev g = geoms[blockIdx.y];
  int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= xb) return;
  const float* bp = bps + g.bp_off;
  const int nk = g.nk, T = g.T, L = g.ray_len;
  int* lo_t = lo + g.lohi_off + bx * nk;
  int* hi_t = hi + g.lohi_off + bx * nk;
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  RayStart r = ray_start(bx, xb, W, T, g.fcos, g.fsin, L);
  int n = 0;
  for (int k = 0; k < nk; ++k) {
    lo_t[k] = INT_MAX;
    hi_t[k] = -1;
  }
  for (int j = 0; j < L; ++j) {
    int ix, iz;
    if (!ray_cell(r, j, W, T, g.fcos, g.fsin, &ix, &iz)) continue;
    float fcount = 0.0f;
    for (int k = 0; k < nk; ++k) {
      int b = cell_bin(ix, iz, W, T, bp[3 * k + 1], bp[3 * k + 2], cent, xb);
      if (b >= 0) fcount = __fadd_rn(fcount, bp[3 * k]);
    }
    if (fcount < 0.001f) continue;
    n++;
    for (int k = 0; k < nk; ++k) {
      int b = cell_bin(ix, iz, W, T, bp[3 * k + 1], bp[3 * k + 2], cent, xb);
      if (b < 0) continue;
      if (b < lo_t[k]) lo_t[k] = b;
      if (b > hi_t[k]) hi_t[k] = b;
    }
  }
  cnt[(size_t)blockIdx.y * xb + bx] = n;
}

// Layout of the operator rows, on the device.  For (tilt i, x-tile t) and each
// neighbour k, the bins touched by the tile's columns are [min lo, max hi]; they
// become consecutive rows of the tile, neighbour after neighbour, and the tile's
// rows are padded to a whole number of kOpChunk (at least one chunk).
// seg[seg_off + t*nk + k] = (row offset within the tile, first bin), segn = its
// row count (0 when the neighbour touches nothing).
__global__ void k_op_tiles(int xb, int ntiles, int n, const OpGeomDev* __restrict__ geoms,
                           const int* __restrict__ lo, const int* __restrict__ hi,
                           int2* __restrict__ seg, int* __restrict__ segn,
                           int* __restrict__ tile_rows, int* __restrict__ tile_used) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n * ntiles) return;
  const int i = q / ntiles, t = q % ntiles;
  const OpGeomDev g = geoms[i];
  const int nk = g.nk;
  const int x0 = t * kOpTileX, x1 = min(xb, x0 + kOpTileX);
  const int* lo_t = lo + g.lohi_off;
  const int* hi_t = hi + g.lohi_off;
  int rows = 0;
  for (int k = 0; k < nk; ++k) {
    int l = INT_MAX, h = -1;
    for (int x = x0; x < x1; ++x) {
      l = min(l, lo_t[(size_t)x * nk + k]);
      h = max(h, hi_t[(size_t)x * nk + k]);
    }
    const size_t e = (size_t)g.seg_off + (size_t)t * nk + k;
    if (h < 0) {
      seg[e] = make_int2(rows, 0);
      segn[e] = 0;
      continue;
    }
    seg[e] = make_int2(rows, l);
    segn[e] = h - l + 1;
    rows += h - l + 1;
  }
  int padded = (rows + kOpChunk - 1) / kOpChunk * kOpChunk;
  if (padded == 0) padded = kOpChunk;
  tile_rows[q] = padded;
  tile_used[q] = rows;
}

// Exclusive prefix sum of count ints in one block of 1024 threads:
// out[j] = sum of in[0..j), out[count] = the total.
__global__ void __launch_bounds__(1024) k_scan_rows(int count, const int* __restrict__ in,
                                                    int* __restrict__ out) {
  __shared__ long long part[1024];
  const int tid = threadIdx.x;
  const int per = (count + 1023) / 1024;
  const int b = min(count, tid * per), e = min(count, b + per);
  long long sum = 0;
  for (int j = b; j < e; ++j) sum += in[j];
  part[tid] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan
    const long long v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  long long run = part[tid] - sum;
  for (int j = b; j < e; ++j) {
    out[j] = (int)run;
    run += in[j];
  }
  if (tid == 1023) out[count] = (int)part[1023];
}

// Per (tilt, x-tile) block: its OpTile and its rows' (tilt, bin) map; padding
// rows point at bin 0 of the first neighbour (their coefficients stay zero).
__global__ void k_op_layout(int ntiles, const OpGeomDev* __restrict__ geoms,
                            const int2* __restrict__ seg, const int* __restrict__ segn,
                            const int* __restrict__ tile_rows, const int* __restrict__ tile_used,
                            const int* __restrict__ row0, OpTile* __restrict__ tiles,
                            int2* __restrict__ rowmap) {
  const int q = blockIdx.x;
  const int i = q / ntiles, t = q % ntiles;
  const OpGeomDev g = geoms[i];
  const int r0 = row0[q], rows = tile_rows[q], used = tile_used[q];
  if (threadIdx.x == 0) {
    OpTile ot;
    ot.row0 = r0;
    ot.rows = rows;
    tiles[q] = ot;
  }
  const size_t e0 = (size_t)g.seg_off + (size_t)t * g.nk;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    int2 m = make_int2(g.i0, 0);
    if (r < used) {
      int k = 0;
      while (k + 1 < g.nk && (segn[e0 + k] == 0 || r >= seg[e0 + k].x + segn[e0 + k])) ++k;
      m = make_int2(g.i0 + k, seg[e0 + k].y + (r - seg[e0 + k].x));
    }
    rowmap[(size_t)r0 + r] = m;
  }
}

// Pass 2: accumulate coefficients.  seg[t*nk + k] = (row offset within the tile,
// first bin).  One thread per (column, neighbour): it owns that column's rows of
// the neighbour's segment, so there are no races and the sums are in ray order.
__global__ void k_op_fill(int xb, const OpGeomDev* __restrict__ geoms,
                          const float* __restrict__ bps, const int* __restrict__ cnt,
                          const OpTile* __restrict__ tiles, const int2* __restrict__ segs,
                          float* __restrict__ coef, int* __restrict__ colvalid) {
  const OpGeomDev g = geoms[blockIdx.z];
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (bx >= xb || k >= g.nk) return;
  const float* bp = bps + g.bp_off;
  const int nk = g.nk, T = g.T, L = g.ray_len;
  const int n = cnt[(size_t)blockIdx.z * xb + bx];
  const bool valid = !((float)n < __fmul_rn(0.8f, (float)L));
  if (k == 0) colvalid[(size_t)blockIdx.z * xb + bx] = valid ? 1 : 0;
  if (!valid) return;
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  const int t = bx / kOpTileX, xl = bx % kOpTileX;
  const OpTile tile = tiles[g.tile_off + t];
  const int2 sg = segs[g.seg_off + t * nk + k];
  const float inv_n = 1.0f / (float)n;
  const float ck = bp[3 * k + 1], sk = bp[3 * k + 2], wk = bp[3 * k];
  float* col = coef + (size_t)tile.row0 * kOpTileX + xl;
  RayStart r = ray_start(bx, xb, W, T, g.fcos, g.fsin, L);
  int cur = -1;
  float acc = 0.0f;
  for (int j = 0; j < L; ++j) {
    int ix, iz;
    if (!ray_cell(r, j, W, T, g.fcos, g.fsin, &ix, &iz)) continue;
    int bk = cell_bin(ix, iz, W, T, ck, sk, cent, xb);
    if (bk < 0) continue;
    float fcount = 0.0f;
    for (int q = 0; q < nk; ++q) {
      int b = cell_bin(ix, iz, W, T, bp[3 * q + 1], bp[3 * q + 2], cent, xb);
      if (b >= 0) fcount = __fadd_rn(fcount, bp[3 * q]);
    }
    if (fcount < 0.001f) continue;
    if (bk != cur) {
      if (cur >= 0) col[(size_t)(sg.x + cur - sg.y) * kOpTileX] += acc;
      cur = bk;
      acc = 0.0f;
    }
    acc += ck * wk / fcount * inv_n;
  }
  if (cur >= 0) col[(size_t)(sg.x + cur - sg.y) * kOpTileX] += acc;
}

int build_reproj_ops(Context* c, const std::vector<ReprojGeom>& geoms, ReprojOpSet* set,
                     cudaStream_t st) {
  const int n = (int)geoms.size();
  set->ops.clear();
  set->bytes = 0;
  set->fma = 0;
  if (n == 0) return MF_OK;
  const int xb = geoms[0].xb, yb = geoms[0].yb;
  const int ntiles = (xb + kOpTileX - 1) / kOpTileX;
  std::vector<OpGeomDev> gd(n);
  std::vector<float> bps;
  int lohi = 0, nkmax = 0;
  size_t nseg = 0;
  for (int i = 0; i < n; ++i) {
    const ReprojGeom& g = geoms[i];
    gd[i].nk = g.nk;
    gd[i].ray_len = g.ray_len;
    gd[i].T = g.thick;
    gd[i].bp_off = (int)bps.size();
    gd[i].fcos = g.fcos;
    gd[i].fsin = g.fsin;
    gd[i].lohi_off = lohi;
    gd[i].tile_off = i * ntiles;
    gd[i].seg_off = (int)nseg;
    gd[i].i0 = g.i0;
    bps.insert(bps.end(), g.bp.begin(), g.bp.end());
    lohi += xb * g.nk;
    nseg += (size_t)ntiles * g.nk;
    nkmax = std::max(nkmax, g.nk);
  }
  const int nt_all = n * ntiles;
  DevBuf d_geom, d_bp, d_cnt, d_lo, d_hi, d_seg, d_segn, d_trows, d_tused, d_row0;
  MF_TRY(d_geom.alloc(sizeof(OpGeomDev) * n));
  MF_TRY(d_bp.alloc(sizeof(float) * bps.size()));
  MF_TRY(d_cnt.alloc(sizeof(int) * (size_t)n * xb));
  MF_TRY(d_lo.alloc(sizeof(int) * (size_t)lohi));
  MF_TRY(d_hi.alloc(sizeof(int) * (size_t)lohi));
  MF_TRY(d_seg.alloc(sizeof(int2) * std::max<size_t>(nseg, 1)));
  MF_TRY(d_segn.alloc(sizeof(int) * std::max<size_t>(nseg, 1)));
  MF_TRY(d_trows.alloc(sizeof(int) * nt_all));
  MF_TRY(d_tused.alloc(sizeof(int) * nt_all));
  MF_TRY(d_row0.alloc(sizeof(int) * (nt_all + 1)));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_geom.p, gd.data(), sizeof(OpGeomDev) * n,
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_bp.p, bps.data(), sizeof(float) * bps.size(),
                                cudaMemcpyHostToDevice, st));
  k_op_scan<<<dim3((xb + 127) / 128, n), 128, 0, st>>>(xb, d_geom.as<OpGeomDev>(),
                                                       d_bp.as<float>(), d_cnt.as<int>(),
                                                       d_lo.as<int>(), d_hi.as<int>());
  k_op_tiles<<<(nt_all + 127) / 128, 128, 0, st>>>(
      xb, ntiles, n, d_geom.as<OpGeomDev>(), d_lo.as<int>(), d_hi.as<int>(), d_seg.as<int2>(),
      d_segn.as<int>(), d_trows.as<int>(), d_tused.as<int>());
  k_scan_rows<<<1, 1024, 0, st>>>(nt_all, d_trows.as<int>(), d_row0.as<int>());
  c->launches += 3;
  MF_CHECK_CUDA(cudaGetLastError());
  // the host needs only the row offsets (allocation size, per-tilt row counts)
  std::vector<int> row0(nt_all + 1);
  MF_CHECK_CUDA(cudaMemcpyAsync(row0.data(), d_row0.p, sizeof(int) * (nt_all + 1),
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  const int total = row0[nt_all];
  for (int i = 0; i < n; ++i) {
    const ReprojGeom& g = geoms[i];
    ReprojOpView v;
    v.ip = g.ip;
    v.i0 = g.i0;
    v.nk = g.nk;
    v.xb = xb;
    v.yb = yb;
    v.ntiles = ntiles;
    v.total_rows = row0[(i + 1) * ntiles] - row0[i * ntiles];
    set->ops.push_back(v);
    set->bytes += 4.0 * (double)xb * yb * (g.nk + 1) + (double)v.total_rows * (kOpTileX * 4 + 8);
    set->fma += (double)yb * v.total_rows * kOpTileX;
  }
  MF_TRY(set->coef.alloc(sizeof(float) * (size_t)total * kOpTileX));
  MF_TRY(set->rowmap.alloc(sizeof(int2) * (size_t)total));
  MF_TRY(set->tiles.alloc(sizeof(OpTile) * nt_all));
  MF_TRY(set->colvalid.alloc(sizeof(int) * (size_t)n * xb));
  MF_CHECK_CUDA(cudaMemsetAsync(set->coef.p, 0, sizeof(float) * (size_t)total * kOpTileX, st));
  k_op_layout<<<nt_all, 128, 0, st>>>(ntiles, d_geom.as<OpGeomDev>(), d_seg.as<int2>(),
                                      d_segn.as<int>(), d_trows.as<int>(), d_tused.as<int>(),
                                      d_row0.as<int>(), set->tiles.as<OpTile>(),
                                      set->rowmap.as<int2>());
  k_op_fill<<<dim3((xb + 127) / 128, nkmax, n), 128, 0, st>>>(
      xb, d_geom.as<OpGeomDev>(), d_bp.as<float>(), d_cnt.as<int>(), set->tiles.as<OpTile>(),
      d_seg.as<int2>(), set->coef.as<float>(), set->colvalid.as<int>());
  c->launches += 2;
  MF_CHECK_CUDA(cudaGetLastError());
  for (int i = 0; i < n; ++i) {
    ReprojOpView& v = set->ops[i];
    v.coef = set->coef.as<float>();
    v.rowmap = set->rowmap.as<int2>();
    v.tiles = set->tiles.as<OpTile>() + (size_t)i * ntiles;
    v.colvalid = set->colvalid.as<int>() + (size_t)i * xb;
  }
  // the temporaries are freed when this returns; wait for the kernels using them
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Tensor-core operator build.  The band of every (x-tile, neighbour) comes from
// the same scan as above; the coefficients are accumulated in FP32 into a
// staging buffer laid out like the final operator (chunk-major, K-major inside a
// chunk), then rounded once to 16 bits.  Held-out tilts are processed in groups
// so that the FP32 staging buffer stays small.
struct TcFillGeom {
  int nk, ray_len, T, bp_off;
  float fcos, fsin;
  int cnt_off;     // int offset of this tilt's per-column valid-sample counts
  int segidx_off;  // int offset of this tilt's (x-tile, neighbour) -> segment table
  int chunk_base;  // first chunk of the staging buffer's window
  int cv_off;      // int offset of this tilt's colvalid entries
};

__global__ void k_optc_fill(int xb, const TcFillGeom* __restrict__ geoms,
                            const float* __restrict__ bps, const int* __restrict__ cnt,
                            const int* __restrict__ segidx, const TcSeg* __restrict__ segs,
                            float* __restrict__ stage, int* __restrict__ colvalid) {
  const TcFillGeom g = geoms[blockIdx.z];
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (bx >= xb || k >= g.nk) return;
  const float* bp = bps + g.bp_off;
  const int nk = g.nk, T = g.T, L = g.ray_len;
  const int n = cnt[g.cnt_off + bx];
  const bool valid = !((float)n < __fmul_rn(0.8f, (float)L));
  if (k == 0) colvalid[g.cv_off + bx] = valid ? 1 : 0;
  if (!valid) return;
  const int t = bx / kTcM, m = bx % kTcM;
  const int si = segidx[g.segidx_off + t * nk + k];
  if (si < 0) return;
  const TcSeg sg = segs[si];
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  const float inv_n = 1.0f / (float)n;
  const float ck = bp[3 * k + 1], sk = bp[3 * k + 2], wk = bp[3 * k];
  float* base = stage + ((size_t)(sg.chunk0 - g.chunk_base) * kTcM + m) * kTcK;
  RayStart r = ray_start(bx, xb, W, T, g.fcos, g.fsin, L);
  int cur = -1;
  float acc = 0.0f;
  auto flush = [&]() {
    const int d = cur - sg.b0;
    base[(size_t)(d / kTcK) * kTcM * kTcK + (d % kTcK)] += acc;
  };
  for (int j = 0; j < L; ++j) {
    int ix, iz;
    if (!ray_cell(r, j, W, T, g.fcos, g.fsin, &ix, &iz)) continue;
    int bk = cell_bin(ix, iz, W, T, ck, sk, cent, xb);
    if (bk < 0) continue;
    float fcount = 0.0f;
    for (int q = 0; q < nk; ++q) {
      int b = cell_bin(ix, iz, W, T, bp[3 * q + 1], bp[3 * q + 2], cent, xb);
      if (b >= 0) fcount = __fadd_rn(fcount, bp[3 * q]);
    }
    if (fcount < 0.001f) continue;
    if (bk != cur) {
      if (cur >= 0) flush();
      cur = bk;
      acc = 0.0f;
    }
    acc += ck * wk / fcount * inv_n;
  }
  if (cur >= 0) flush();
}

__global__ void k_op_to_fp16(const float* __restrict__ src, size_t n, float scale,
                             __half* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __float2half_rn(src[i] * scale);
}
__global__ void k_op_to_bf16(const float* __restrict__ src, size_t n, float scale,
                             __nv_bfloat16* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i] * scale);
}

// Segment table of the tensor-core operators, on the device.  Entry (tilt i,
// x-tile t, neighbour k), flattened in that order from the tilt's segidx_off:
// the bins [min lo, max hi] of the tile's columns become a segment from b0 = lo
// rounded down to a multiple of 8, of nch chunks of kTcK bins (none when the
// neighbour touches nothing).
__global__ void k_optc_tiles(int xb, int ntx, int n, const OpGeomDev* __restrict__ geoms,
                             const int* __restrict__ lo, const int* __restrict__ hi,
                             int* __restrict__ ent_b0, int* __restrict__ ent_nch,
                             int* __restrict__ ent_seg) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n * ntx) return;
  const int i = q / ntx, t = q % ntx;
  const OpGeomDev g = geoms[i];
  const int nk = g.nk;
  const int x0 = t * kTcM, x1 = min(xb, x0 + kTcM);
  const int* lo_t = lo + g.lohi_off;
  const int* hi_t = hi + g.lohi_off;
  for (int k = 0; k < nk; ++k) {
    int l = INT_MAX, h = -1;
    for (int x = x0; x < x1; ++x) {
      l = min(l, lo_t[(size_t)x * nk + k]);
      h = max(h, hi_t[(size_t)x * nk + k]);
    }
    const size_t e = (size_t)g.seg_off + (size_t)t * nk + k;
    const int b0 = l & ~7;
    ent_b0[e] = h < 0 ? 0 : b0;
    ent_nch[e] = h < 0 ? 0 : (h - b0 + kTcK) / kTcK;
    ent_seg[e] = h < 0 ? 0 : 1;
  }
}

// From the entries and their exclusive prefix sums (segment index, first chunk):
// segidx (-1 for an empty entry), the segments, and every x-tile's summary.
__global__ void k_optc_layout(int ntx, const OpGeomDev* __restrict__ geoms,
                              const int* __restrict__ ent_b0, const int* __restrict__ ent_nch,
                              const int* __restrict__ ent_seg, const int* __restrict__ seg_pre,
                              const int* __restrict__ chunk_pre, int* __restrict__ segidx,
                              TcSeg* __restrict__ segs, TcXTile* __restrict__ xts) {
  const int i = blockIdx.x;
  const OpGeomDev g = geoms[i];
  const int nk = g.nk, ne = ntx * nk;
  for (int j = threadIdx.x; j < ne; j += blockDim.x) {
    const size_t e = (size_t)g.seg_off + j;
    if (ent_seg[e]) {
      TcSeg sg;
      sg.tilt = g.i0 + j % nk;
      sg.b0 = ent_b0[e];
      sg.nch = ent_nch[e];
      sg.chunk0 = chunk_pre[e];
      segs[seg_pre[e]] = sg;
      segidx[e] = seg_pre[e];
    } else {
      segidx[e] = -1;
    }
  }
  for (int t = threadIdx.x; t < ntx; t += blockDim.x) {
    const size_t e0 = (size_t)g.seg_off + (size_t)t * nk, e1 = e0 + nk;
    TcXTile X;
    X.seg0 = seg_pre[e0];
    X.nseg = seg_pre[e1] - seg_pre[e0];
    X.nch = chunk_pre[e1] - chunk_pre[e0];
    X.pad = 0;
    xts[(size_t)i * ntx + t] = X;
  }
}

int build_reproj_tc_ops(Context* c, const std::vector<ReprojGeom>& geoms, int half_kind,
                        TcOpSet* set, cudaStream_t st) {
  const int n = (int)geoms.size();
  set->ops.clear();
  set->bytes = 0;
  set->fma = 0;
  set->total_chunks = 0;
  set->half_kind = half_kind;
  if (half_kind != MF_PREC_BF16 && half_kind != MF_PREC_FP16)
    return set_error(MF_ERR_ARG, "tensor-core operators need FP16 or BF16 (got %d)", half_kind);
  if (n == 0) return MF_OK;
  const int xb = geoms[0].xb, yb = geoms[0].yb;
  const int ntx = (xb + kTcM - 1) / kTcM;
  // pass 1: per column valid-sample count and per neighbour bin range; then the
  // segment table, laid out on the device (the host reads back only prefix sums)
  std::vector<OpGeomDev> gd(n);
  std::vector<float> bps;
  int lohi = 0;
  std::vector<int> segidx_off(n);
  size_t nent = 0;
  for (int i = 0; i < n; ++i) {
    const ReprojGeom& g = geoms[i];
    gd[i].nk = g.nk;
    gd[i].ray_len = g.ray_len;
    gd[i].T = g.thick;
    gd[i].bp_off = (int)bps.size();
    gd[i].fcos = g.fcos;
    gd[i].fsin = g.fsin;
    gd[i].lohi_off = lohi;
    gd[i].tile_off = 0;
    gd[i].seg_off = (int)nent;
    gd[i].i0 = g.i0;
    segidx_off[i] = (int)nent;
    bps.insert(bps.end(), g.bp.begin(), g.bp.end());
    lohi += xb * g.nk;
    nent += (size_t)ntx * g.nk;
  }
  DevBuf d_geom, d_bp, d_cnt, d_lo, d_hi, d_b0, d_nch, d_has, d_segpre, d_chpre;
  MF_TRY(d_geom.alloc(sizeof(OpGeomDev) * n));
  MF_TRY(d_bp.alloc(sizeof(float) * bps.size()));
  MF_TRY(d_cnt.alloc(sizeof(int) * (size_t)n * xb));
  MF_TRY(d_lo.alloc(sizeof(int) * (size_t)lohi));
  MF_TRY(d_hi.alloc(sizeof(int) * (size_t)lohi));
  MF_TRY(d_b0.alloc(sizeof(int) * std::max<size_t>(nent, 1)));
  MF_TRY(d_nch.alloc(sizeof(int) * std::max<size_t>(nent, 1)));
  MF_TRY(d_has.alloc(sizeof(int) * std::max<size_t>(nent, 1)));
  MF_TRY(d_segpre.alloc(sizeof(int) * (nent + 1)));
  MF_TRY(d_chpre.alloc(sizeof(int) * (nent + 1)));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_geom.p, gd.data(), sizeof(OpGeomDev) * n,
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_bp.p, bps.data(), sizeof(float) * bps.size(),
                                cudaMemcpyHostToDevice, st));
  k_op_scan<<<dim3((xb + 127) / 128, n), 128, 0, st>>>(xb, d_geom.as<OpGeomDev>(),
                                                       d_bp.as<float>(), d_cnt.as<int>(),
                                                       d_lo.as<int>(), d_hi.as<int>());
  k_optc_tiles<<<(n * ntx + 127) / 128, 128, 0, st>>>(
      xb, ntx, n, d_geom.as<OpGeomDev>(), d_lo.as<int>(), d_hi.as<int>(), d_b0.as<int>(),
      d_nch.as<int>(), d_has.as<int>());
  k_scan_rows<<<1, 1024, 0, st>>>((int)nent, d_has.as<int>(), d_segpre.as<int>());
  k_scan_rows<<<1, 1024, 0, st>>>((int)nent, d_nch.as<int>(), d_chpre.as<int>());
  c->launches += 4;
  MF_CHECK_CUDA(cudaGetLastError());
  std::vector<int> chpre(nent + 1), segpre_end(1);
  MF_CHECK_CUDA(cudaMemcpyAsync(chpre.data(), d_chpre.p, sizeof(int) * (nent + 1),
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(segpre_end.data(), d_segpre.as<int>() + nent, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  std::vector<int> chunk_first(n + 1);
  for (int i = 0; i < n; ++i) chunk_first[i] = chpre[segidx_off[i]];
  chunk_first[n] = chpre[nent];
  const int chunks = chunk_first[n];
  for (int i = 0; i < n; ++i) {
    const ReprojGeom& g = geoms[i];
    TcOpView v;
    v.ip = g.ip;
    v.i0 = g.i0;
    v.nk = g.nk;
    v.xb = xb;
    v.yb = yb;
    v.ntx = ntx;
    v.nchunks = chunk_first[i + 1] - chunk_first[i];
    set->ops.push_back(v);
    // compulsory traffic: 16-bit neighbour images, FP32 output, the operator itself
    set->bytes += 2.0 * xb * yb * g.nk + 4.0 * xb * yb + (double)v.nchunks * kTcM * kTcK * 2;
    set->fma += (double)v.nchunks * kTcM * kTcK * yb;
  }
  set->total_chunks = chunks;
  set->nsegs = segpre_end[0];
  set->nxt = n * ntx;
  const size_t chunk_elems = (size_t)kTcM * kTcK;
  MF_TRY(set->op16.alloc(2 * chunk_elems * std::max(chunks, 1)));
  MF_TRY(set->xt.alloc(sizeof(TcXTile) * (size_t)n * ntx));
  MF_TRY(set->segs.alloc(sizeof(TcSeg) * std::max(set->nsegs, 1)));
  MF_TRY(set->colvalid.alloc(sizeof(int) * (size_t)n * xb));
  DevBuf d_segidx;
  MF_TRY(d_segidx.alloc(sizeof(int) * std::max<size_t>(nent, 1)));
  k_optc_layout<<<n, 256, 0, st>>>(ntx, d_geom.as<OpGeomDev>(), d_b0.as<int>(), d_nch.as<int>(),
                                   d_has.as<int>(), d_segpre.as<int>(), d_chpre.as<int>(),
                                   d_segidx.as<int>(), set->segs.as<TcSeg>(),
                                   set->xt.as<TcXTile>());
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  // pass 2 in groups of tilts whose FP32 staging fits in a bounded buffer
  const size_t stage_cap = (size_t)64 << 20;  // floats (256 MB)
  size_t max_one = 0;
  for (int i = 0; i < n; ++i)
    max_one = std::max(max_one, (size_t)(chunk_first[i + 1] - chunk_first[i]) * chunk_elems);
  DevBuf stagebuf, d_fg;
  MF_TRY(stagebuf.alloc(sizeof(float) * std::max(std::min(stage_cap, (size_t)chunks * chunk_elems),
                                                  std::max<size_t>(max_one, 1))));
  MF_TRY(d_fg.alloc(sizeof(TcFillGeom) * n));
  std::vector<TcFillGeom> fg(n);
  int nkmax = 0;
  for (int i = 0; i < n; ++i) {
    fg[i].nk = geoms[i].nk;
    fg[i].ray_len = geoms[i].ray_len;
    fg[i].T = geoms[i].thick;
    fg[i].bp_off = gd[i].bp_off;
    fg[i].fcos = geoms[i].fcos;
    fg[i].fsin = geoms[i].fsin;
    fg[i].cnt_off = i * xb;
    fg[i].segidx_off = segidx_off[i];
    fg[i].cv_off = i * xb;
    fg[i].chunk_base = 0;
    nkmax = std::max(nkmax, geoms[i].nk);
  }
  const size_t cap_elems = stagebuf.bytes / sizeof(float);
  int g0 = 0;
  while (g0 < n) {
    int g1 = g0 + 1;
    while (g1 < n && (size_t)(chunk_first[g1 + 1] - chunk_first[g0]) * chunk_elems <= cap_elems)
      ++g1;
    const size_t elems = (size_t)(chunk_first[g1] - chunk_first[g0]) * chunk_elems;
    for (int i = g0; i < g1; ++i) fg[i].chunk_base = chunk_first[g0];
    MF_CHECK_CUDA(cudaMemcpyAsync(d_fg.as<TcFillGeom>() + g0, fg.data() + g0,
                                  sizeof(TcFillGeom) * (g1 - g0), cudaMemcpyHostToDevice, st));
    if (elems > 0) MF_CHECK_CUDA(cudaMemsetAsync(stagebuf.p, 0, sizeof(float) * elems, st));
    k_optc_fill<<<dim3((xb + 127) / 128, nkmax, g1 - g0), 128, 0, st>>>(
        xb, d_fg.as<TcFillGeom>() + g0, d_bp.as<float>(), d_cnt.as<int>(), d_segidx.as<int>(),
        set->segs.as<TcSeg>(), stagebuf.as<float>(), set->colvalid.as<int>());
    c->launches++;
    MF_CHECK_CUDA(cudaGetLastError());
    if (elems > 0) {
      const int blocks = (int)std::min<size_t>((elems + 255) / 256, (size_t)c->sm_count * 16);
      if (half_kind == MF_PREC_FP16)
        k_op_to_fp16<<<blocks, 256, 0, st>>>(
            stagebuf.as<float>(), elems, kTcScale,
            set->op16.as<__half>() + (size_t)chunk_first[g0] * chunk_elems);
      else
        k_op_to_bf16<<<blocks, 256, 0, st>>>(
            stagebuf.as<float>(), elems, kTcScale,
            set->op16.as<__nv_bfloat16>() + (size_t)chunk_first[g0] * chunk_elems);
      c->launches++;
      MF_CHECK_CUDA(cudaGetLastError());
    }
    g0 = g1;
  }
  for (int i = 0; i < n; ++i) {
    TcOpView& v = set->ops[i];
    v.xt = set->xt.as<TcXTile>() + (size_t)i * ntx;
    v.segs = set->segs.as<TcSeg>();
    v.colvalid = set->colvalid.as<int>() + (size_t)i * xb;
  }
  MF_TRY(tc_op_map(set));
  // the temporaries are freed when this returns; wait for the kernels using them
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Operators for geometries of several image sizes: one set per size, concatenated.
static std::vector<std::vector<int>> split_by_shape(const std::vector<ReprojGeom>& geoms) {
  std::vector<std::vector<int>> parts;
  std::vector<std::pair<int, int>> shapes;
  for (int i = 0; i < (int)geoms.size(); ++i) {
    const std::pair<int, int> sh(geoms[i].xb, geoms[i].yb);
    size_t k = 0;
    while (k < shapes.size() && shapes[k] != sh) ++k;
    if (k == shapes.size()) {
      shapes.push_back(sh);
      parts.emplace_back();
    }
    parts[k].push_back(i);
  }
  return parts;
}

int build_reproj_ops_any(Context* c, const std::vector<ReprojGeom>& geoms, ReprojOpSet* set,
                         cudaStream_t st) {
  const auto parts = split_by_shape(geoms);
  if (parts.size() <= 1) return build_reproj_ops(c, geoms, set, st);
  std::vector<ReprojOpSet> sub(parts.size());
  size_t rows = 0, ntile = 0, ncv = 0;
  std::vector<size_t> row_off, tile_off, cv_off;
  for (size_t p = 0; p < parts.size(); ++p) {
    std::vector<ReprojGeom> g;
    for (int i : parts[p]) g.push_back(geoms[i]);
    MF_TRY(build_reproj_ops(c, g, &sub[p], st));
    row_off.push_back(rows);
    tile_off.push_back(ntile);
    cv_off.push_back(ncv);
    for (const ReprojOpView& v : sub[p].ops) rows += v.total_rows;
    ntile += (size_t)sub[p].ops.size() * sub[p].ops[0].ntiles;
    ncv += (size_t)sub[p].ops.size() * sub[p].ops[0].xb;
  }
  MF_TRY(set->coef.alloc(sizeof(float) * rows * kOpTileX));
  MF_TRY(set->rowmap.alloc(sizeof(int2) * rows));
  MF_TRY(set->tiles.alloc(sizeof(OpTile) * ntile));
  MF_TRY(set->colvalid.alloc(sizeof(int) * ncv));
  set->ops.assign(geoms.size(), ReprojOpView());
  set->bytes = 0;
  set->fma = 0;
  for (size_t p = 0; p < parts.size(); ++p) {
    const ReprojOpSet& q = sub[p];
    size_t prow = 0;
    for (const ReprojOpView& v : q.ops) prow += v.total_rows;
    const int nt = q.ops[0].ntiles, xb = q.ops[0].xb;
    const size_t pt = q.ops.size() * (size_t)nt;
    MF_CHECK_CUDA(cudaMemcpyAsync(set->coef.as<float>() + row_off[p] * kOpTileX, q.coef.p,
                                  sizeof(float) * prow * kOpTileX, cudaMemcpyDeviceToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(set->rowmap.as<int2>() + row_off[p], q.rowmap.p,
                                  sizeof(int2) * prow, cudaMemcpyDeviceToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(set->colvalid.as<int>() + cv_off[p], q.colvalid.p,
                                  sizeof(int) * q.ops.size() * xb, cudaMemcpyDeviceToDevice, st));
    std::vector<OpTile> t(pt);
    MF_CHECK_CUDA(cudaMemcpyAsync(t.data(), q.tiles.p, sizeof(OpTile) * pt,
                                  cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaStreamSynchronize(st));
    for (OpTile& x : t) x.row0 += (int)row_off[p];
    MF_CHECK_CUDA(cudaMemcpyAsync(set->tiles.as<OpTile>() + tile_off[p], t.data(),
                                  sizeof(OpTile) * pt, cudaMemcpyHostToDevice, st));
    for (size_t li = 0; li < parts[p].size(); ++li) {
      ReprojOpView v = q.ops[li];
      v.coef = set->coef.as<float>();
      v.rowmap = set->rowmap.as<int2>();
      v.tiles = set->tiles.as<OpTile>() + tile_off[p] + li * nt;
      v.colvalid = set->colvalid.as<int>() + cv_off[p] + li * xb;
      set->ops[parts[p][li]] = v;
    }
    set->bytes += q.bytes;
    set->fma += q.fma;
  }
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

int build_reproj_tc_ops_any(Context* c, const std::vector<ReprojGeom>& geoms, int half_kind,
                            TcOpSet* set, cudaStream_t st) {
  const auto parts = split_by_shape(geoms);
  if (parts.size() <= 1) return build_reproj_tc_ops(c, geoms, half_kind, set, st);
  std::vector<TcOpSet> sub(parts.size());
  int chunks = 0, nsegs = 0, nxt = 0;
  size_t ncv = 0;
  std::vector<int> chunk_off, seg_off, xt_off;
  std::vector<size_t> cv_off;
  for (size_t p = 0; p < parts.size(); ++p) {
    std::vector<ReprojGeom> g;
    for (int i : parts[p]) g.push_back(geoms[i]);
    MF_TRY(build_reproj_tc_ops(c, g, half_kind, &sub[p], st));
    chunk_off.push_back(chunks);
    seg_off.push_back(nsegs);
    xt_off.push_back(nxt);
    cv_off.push_back(ncv);
    chunks += sub[p].total_chunks;
    nsegs += sub[p].nsegs;
    nxt += sub[p].nxt;
    ncv += sub[p].ops.size() * (size_t)sub[p].ops[0].xb;
  }
  const size_t chunk_bytes = (size_t)kTcM * kTcK * 2;
  MF_TRY(set->op16.alloc(chunk_bytes * std::max(chunks, 1)));
  MF_TRY(set->segs.alloc(sizeof(TcSeg) * std::max(nsegs, 1)));
  MF_TRY(set->xt.alloc(sizeof(TcXTile) * std::max(nxt, 1)));
  MF_TRY(set->colvalid.alloc(sizeof(int) * ncv));
  set->ops.assign(geoms.size(), TcOpView());
  set->total_chunks = chunks;
  set->nsegs = nsegs;
  set->nxt = nxt;
  set->half_kind = half_kind;
  set->bytes = 0;
  set->fma = 0;
  for (size_t p = 0; p < parts.size(); ++p) {
    const TcOpSet& q = sub[p];
    const int ntx = q.ops[0].ntx, xb = q.ops[0].xb;
    if (q.total_chunks > 0)
      MF_CHECK_CUDA(cudaMemcpyAsync((char*)set->op16.p + chunk_bytes * chunk_off[p], q.op16.p,
                                    chunk_bytes * q.total_chunks, cudaMemcpyDeviceToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(set->colvalid.as<int>() + cv_off[p], q.colvalid.p,
                                  sizeof(int) * q.ops.size() * xb, cudaMemcpyDeviceToDevice, st));
    std::vector<TcSeg> sg(q.nsegs);
    std::vector<TcXTile> xt(q.nxt);
    if (q.nsegs > 0)
      MF_CHECK_CUDA(cudaMemcpyAsync(sg.data(), q.segs.p, sizeof(TcSeg) * q.nsegs,
                                    cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(xt.data(), q.xt.p, sizeof(TcXTile) * q.nxt,
                                  cudaMemcpyDeviceToHost, st));
    MF_CHECK_CUDA(cudaStreamSynchronize(st));
    for (TcSeg& x : sg) x.chunk0 += chunk_off[p];
    for (TcXTile& x : xt) x.seg0 += seg_off[p];
    if (q.nsegs > 0)
      MF_CHECK_CUDA(cudaMemcpyAsync(set->segs.as<TcSeg>() + seg_off[p], sg.data(),
                                    sizeof(TcSeg) * q.nsegs, cudaMemcpyHostToDevice, st));
    MF_CHECK_CUDA(cudaMemcpyAsync(set->xt.as<TcXTile>() + xt_off[p], xt.data(),
                                  sizeof(TcXTile) * q.nxt, cudaMemcpyHostToDevice, st));
    for (size_t li = 0; li < parts[p].size(); ++li) {
      TcOpView v = q.ops[li];
      v.xt = set->xt.as<TcXTile>() + xt_off[p] + li * ntx;
      v.segs = set->segs.as<TcSeg>();
      v.colvalid = set->colvalid.as<int>() + cv_off[p] + li * xb;
      set->ops[parts[p][li]] = v;
    }
    set->bytes += q.bytes;
    set->fma += q.fma;
  }
  MF_TRY(tc_op_map(set));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// Packed FP32 pairs for fma.rn.f32x2 (sm_100): each lane is the scalar IEEE
// fused multiply-add, so a pair of accumulators advances exactly as two fmaf.
__device__ __forceinline__ unsigned long long f2pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 f2unpack(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// ---------------------------------------------------------------------------
// Operator apply: out[y][x] = sum_r A[y][r] * B_t[r][x] with A gathered from the
// neighbour rows through rowmap.  One CTA computes a kApplyTileY x kOpTileX
// (128 x 64) output tile with 256 threads, each an 8 x 4 register tile.  Operator
// rows are consumed kOpChunk at a time through two shared-memory buffers; the
// next chunk's global loads are issued before the current chunk's FMAs, so
// memory latency hides behind arithmetic.  Every loaded neighbour value is
// tested for the -1e30 sentinel; a hit flags the row tile for the exact path.
// The multiply-adds run as packed pairs (fma.rn.f32x2), lane for lane fmaf.
constexpr int kApplyThreads = 256;
constexpr int kAPerThread = kOpChunk * kApplyTileY / kApplyThreads;  // 8

__global__ void __launch_bounds__(kApplyThreads, 2)
    k_op_apply(const float* __restrict__ corr, int xb, int yb, size_t pix,
               const float* __restrict__ coef, const int2* __restrict__ rowmap,
               const OpTile* __restrict__ tiles, const int* __restrict__ colvalid,
               int* __restrict__ rowflags, float* __restrict__ out,
               const ApplyJob* __restrict__ jobs, const int* __restrict__ active) {
  if (jobs) {
    // group form: blockIdx.z selects the series, with its own size
    if (active && active[blockIdx.z] == 0) return;
    const ApplyJob J = jobs[blockIdx.z];
    if ((int)blockIdx.x >= J.ntiles || (int)blockIdx.y * kApplyTileY >= J.yb) return;
    corr = J.corr;
    tiles = J.tiles;
    colvalid = J.colvalid;
    rowflags = J.rowflags;
    out = J.out;
    xb = J.xb;
    yb = J.yb;
    pix = (size_t)J.xb * J.yb;
  }
  __shared__ __align__(16) float As[2][kOpChunk][kApplyTileY];
  __shared__ __align__(16) float Bs[2][kOpChunk][kOpTileX];
  __shared__ int s_flag;
  const int t = blockIdx.x;
  const int y0 = blockIdx.y * kApplyTileY;
  const int x0 = t * kOpTileX;
  const OpTile tile = tiles[t];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;  // 16 x 4 columns, 16 x 8 rows
  if (tid == 0) s_flag = 0;
  unsigned long long acc2[8][2];  // columns 2h, 2h + 1 of row i (packed FMA pairs)
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) acc2[i][h] = 0ull;
  const int lr = tid % kOpChunk;  // operator row this thread loads for A
  const int ly = tid / kOpChunk;  // first y row it loads (then every 16th)
  bool bad = false;
  float ra[kAPerThread];
  float4 rb;
  auto load_chunk = [&](int r0) {
    const int row = tile.row0 + r0;
    const int2 rm = __ldg(rowmap + row + lr);
    const float* src = corr + (size_t)rm.x * pix + rm.y;
#pragma unroll
    for (int q = 0; q < kAPerThread; ++q) {
      const int y = y0 + ly + 16 * q;
      ra[q] = (y < yb) ? __ldg(src + (size_t)y * xb) : 0.0f;
    }
    rb = __ldg(reinterpret_cast<const float4*>(coef + (size_t)row * kOpTileX) + tid);
  };
  auto store_chunk = [&](int buf) {
#pragma unroll
    for (int q = 0; q < kAPerThread; ++q) {
      As[buf][lr][ly + 16 * q] = ra[q];
      bad |= (ra[q] < -1e10f);
    }
    reinterpret_cast<float4*>(&Bs[buf][0][0])[tid] = rb;
  };
  const int nchunks = tile.rows / kOpChunk;
  load_chunk(0);
  store_chunk(0);
  __syncthreads();
  for (int c = 0; c < nchunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < nchunks) load_chunk((c + 1) * kOpChunk);
#pragma unroll
    for (int rr = 0; rr < kOpChunk; ++rr) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][rr][ty * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][rr][ty * 8 + 4]);
      const float4 b = *reinterpret_cast<const float4*>(&Bs[buf][rr][tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const unsigned long long bp[2] = {f2pack(b.x, b.y), f2pack(b.z, b.w)};
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const unsigned long long ap = f2pack(av[i], av[i]);
#pragma unroll
        for (int h = 0; h < 2; ++h) acc2[i][h] = ffma2(ap, bp[h], acc2[i][h]);
      }
    }
    if (c + 1 < nchunks) store_chunk(buf ^ 1);
    __syncthreads();
  }
  float acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float2 v = f2unpack(acc2[i][h]);
      acc[i][2 * h] = v.x;
      acc[i][2 * h + 1] = v.y;
    }
  if (bad) s_flag = 1;
  __syncthreads();
  if (tid == 0 && s_flag) atomicOr(&rowflags[blockIdx.y], 1);
  const int xc = x0 + tx * 4;
  int cv[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) cv[j] = (xc + j < xb) ? colvalid[xc + j] : 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int y = y0 + ty * 8 + i;
    if (y >= yb) continue;
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = cv[j] ? acc[i][j] : kSentinel;
    float* o = out + (size_t)y * xb + xc;
    if (xc + 3 < xb && ((xb & 3) == 0)) {
      *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (xc + j < xb) o[j] = v[j];
    }
  }
}

int launch_reproject_apply(Context* c, const ReprojOpView& op, const float* corr, size_t pix,
                           int* d_rowflags, float* out, cudaStream_t st) {
  dim3 grd(op.ntiles, (op.yb + kApplyTileY - 1) / kApplyTileY);
  k_op_apply<<<grd, 256, 0, st>>>(corr, op.xb, op.yb, pix, op.coef, op.rowmap, op.tiles,
                                  op.colvalid, d_rowflags, out, nullptr, nullptr);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Group form of the FP32 apply, for whole groups of series: a CTA computes 256
// image rows x 64 output columns with 256 threads, each an 8 x 8 register tile
// (rows ty*4..+3 and 128+ty*4..+3, columns tx*4..+3 and 32+tx*4..+3, so that the
// warp's shared-memory reads are contiguous 16-byte vectors).  Operator rows are
// consumed 16 at a time through a 3-stage shared-memory ring fed by cp.async: the
// gathered neighbour values (4-byte copies, zero-filled below the image) and the
// coefficient chunk (16-byte copies) go straight from global to shared memory,
// with no staging registers.  Sentinels are not tested here: the per-(tilt,
// 128-row tile) flags of the corrected stack (k_flag_tiles_group) send the tiles
// whose neighbours hold a -1e30 to the exact path, which overwrites them.
// The multiply-adds run as packed pairs (fma.rn.f32x2, two columns per
// instruction), lane for lane the fmaf of the scalar form in the same order, so
// the output is bit for bit that of one fmaf chain per output over the operator
// rows, with half the FMA instructions to issue.
constexpr int kA2Y = 256;        // image rows per CTA
constexpr int kA2Stages = 3;     // cp.async ring depth (measured best of 2, 3, 4)
constexpr int kA2Pitch = 260;    // floats per operator row of the A tile (256 + 4)
constexpr int kA2SmemBytes = kA2Stages * kOpChunk * (kA2Pitch + kOpTileX) * 4;

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(256, 2)
    k_op_apply_group(const float* __restrict__ coef, const int2* __restrict__ rowmap,
                     const ApplyJob* __restrict__ jobs, const int* __restrict__ active) {
  if (active && active[blockIdx.z] == 0) return;
  const ApplyJob J = jobs[blockIdx.z];
  if ((int)blockIdx.x >= J.ntiles || (int)blockIdx.y * kA2Y >= J.yb) return;
  extern __shared__ __align__(16) float smem[];
  float* As = smem;                                      // [stage][16][kA2Pitch]
  float* Bs = smem + kA2Stages * kOpChunk * kA2Pitch;    // [stage][16][64]
  const int xb = J.xb, yb = J.yb;
  const size_t pix = (size_t)xb * yb;
  const int y0 = blockIdx.y * kA2Y;
  const int x0 = blockIdx.x * kOpTileX;
  const OpTile tile = J.tiles[blockIdx.x];
  const int nchunks = tile.rows / kOpChunk;
  const int tid = threadIdx.x;
  const int lr = tid % kOpChunk, ly = tid / kOpChunk;  // loader: operator row, first image row
  const uint32_t as_base = (uint32_t)__cvta_generic_to_shared(As);
  const uint32_t bs_base = (uint32_t)__cvta_generic_to_shared(Bs);
  auto load = [&](int c) {
    const int st = c % kA2Stages;
    const int row = tile.row0 + c * kOpChunk;
    const int2 rm = __ldg(rowmap + row + lr);
    const float* src = J.corr + (size_t)rm.x * pix + rm.y;
    const uint32_t a = as_base + (uint32_t)((st * kOpChunk + lr) * kA2Pitch) * 4u;
#pragma unroll
    for (int q = 0; q < kA2Y / 16; ++q) {
      const int y = ly + 16 * q;
      const bool in = y0 + y < yb;
      cp_async4(a + (uint32_t)y * 4u, in ? src + (size_t)(y0 + y) * xb : src, in);
    }
    cp_async16(bs_base + (uint32_t)(st * kOpChunk * kOpTileX + tid * 4) * 4u,
               coef + (size_t)row * kOpTileX + tid * 4);
  };
  const int tx = tid % 8, ty = tid / 8;
  // acc2[i][h] holds the accumulators of columns 2h and 2h + 1 of row i
  unsigned long long acc2[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int h = 0; h < 4; ++h) acc2[i][h] = 0ull;
#pragma unroll
  for (int c = 0; c < kA2Stages - 1; ++c) {
    if (c < nchunks) load(c);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<kA2Stages - 2>();
    __syncthreads();
    if (c + kA2Stages - 1 < nchunks) load(c + kA2Stages - 1);
    cp_async_commit();
    const float* A = As + (c % kA2Stages) * kOpChunk * kA2Pitch;
    const float* Bt = Bs + (c % kA2Stages) * kOpChunk * kOpTileX;
#pragma unroll
    for (int rr = 0; rr < kOpChunk; ++rr) {
      const float4 a0 = *reinterpret_cast<const float4*>(A + rr * kA2Pitch + ty * 4);
      const float4 a1 = *reinterpret_cast<const float4*>(A + rr * kA2Pitch + 128 + ty * 4);
      const float4 b0 = *reinterpret_cast<const float4*>(Bt + rr * kOpTileX + tx * 4);
      const float4 b1 = *reinterpret_cast<const float4*>(Bt + rr * kOpTileX + 32 + tx * 4);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const unsigned long long bp[4] = {f2pack(b0.x, b0.y), f2pack(b0.z, b0.w),
                                        f2pack(b1.x, b1.y), f2pack(b1.z, b1.w)};
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const unsigned long long ap = f2pack(av[i], av[i]);
#pragma unroll
        for (int h = 0; h < 4; ++h) acc2[i][h] = ffma2(ap, bp[h], acc2[i][h]);
      }
    }
  }
  cp_async_wait<0>();
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const float2 v = f2unpack(acc2[i][h]);
      acc[i][2 * h] = v.x;
      acc[i][2 * h + 1] = v.y;
    }
  int cv[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int x = x0 + (j < 4 ? tx * 4 + j : 32 + tx * 4 + j - 4);
    cv[j] = x < xb ? J.colvalid[x] : 0;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int y = y0 + (i < 4 ? ty * 4 + i : 128 + ty * 4 + i - 4);
    if (y >= yb) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int xc = x0 + h * 32 + tx * 4;
      float v[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = cv[4 * h + j] ? acc[i][4 * h + j] : kSentinel;
      float* o = J.out + (size_t)y * xb + xc;
      if (xc + 3 < xb && (xb & 3) == 0) {
        *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (xc + j < xb) o[j] = v[j];
      }
    }
  }
}

// The group apply's shared-memory size, set once per device outside any stream
// capture (the set-up of a pass calls it before the pass is captured).
int prepare_apply_group(Context* c) {
  // per device ordinal; serving workers may get here at the same time (setting the
  // attribute twice is harmless, the flag only saves the call)
  static std::atomic<bool> attr_set[64] = {};
  if (!attr_set[c->gpu & 63].load(std::memory_order_acquire)) {
    MF_CHECK_CUDA(cudaFuncSetAttribute(k_op_apply_group,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kA2SmemBytes));
    attr_set[c->gpu & 63].store(true, std::memory_order_release);
  }
  return MF_OK;
}

int launch_reproject_apply_group(Context* c, const ReprojOpSet& set, const ApplyJob* d_jobs,
                                 const int* active, int njobs, int ntiles_max, int yb_max,
                                 cudaStream_t st) {
  MF_TRY(prepare_apply_group(c));
  dim3 grd(ntiles_max, (yb_max + kA2Y - 1) / kA2Y, njobs);
  k_op_apply_group<<<grd, 256, kA2SmemBytes, st>>>(set.coef.as<float>(), set.rowmap.as<int2>(),
                                                   d_jobs, active);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// Per-(tilt, 128-row tile, column part) flags of an FP32 corrected stack: set when
// the piece holds a -1e30 sentinel (the banded operator cannot carry one; the exact
// path then recomputes every output tile that reads it).  All tilts of every
// series (steps == null) or each series' held-out tilt of a step.
__global__ void k_flag_tiles_group(const GroupSeriesDev* __restrict__ ser,
                                   const GroupStepDev* __restrict__ steps,
                                   const int* __restrict__ active, int nz_max) {
  const int j = blockIdx.z;
  const int b = steps ? j : j / nz_max;
  if (active && active[b] == 0) return;
  const GroupSeriesDev& S = ser[b];
  const int tz = steps ? steps[b].ip : j % nz_max;
  if (tz < 0 || tz >= S.nz || (int)blockIdx.y >= S.ytiles) return;
  const int xb = S.xb, yb = S.yb;
  const float* s = S.corr + (size_t)tz * xb * yb;
  const int ya = blockIdx.y * kApplyTileY, yz = min(yb, ya + kApplyTileY);
  const int half_x = xb / 2;
  const int p0 = half_x * blockIdx.x / kFlagParts, p1 = half_x * (blockIdx.x + 1) / kFlagParts;
  int bad = 0;
#pragma unroll 4  // several rows' loads in flight per thread
  for (int y = ya + threadIdx.y; y < yz; y += blockDim.y) {
    const float2* row = reinterpret_cast<const float2*>(s + (size_t)y * xb);
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
      const float2 v = row[p];
      bad |= (v.x < -1e10f) | (v.y < -1e10f);
    }
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    S.tflags[((size_t)tz * S.ytiles + blockIdx.y) * kFlagParts + blockIdx.x] = bad ? 1 : 0;
}

int launch_flag_tiles_group(Context* c, const GroupSeriesDev* ser, const GroupStepDev* steps,
                            const int* active, int nseries, int nz_max, int ytiles_max,
                            cudaStream_t st) {
  if (nseries <= 0) return MF_OK;
  dim3 blk(64, 8), grd(kFlagParts, ytiles_max, steps ? nseries : nseries * nz_max);
  k_flag_tiles_group<<<grd, blk, 0, st>>>(ser, steps, active, nz_max);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// The same flags for one series' corrected stack: every tilt (tilts == null) or
// the tilts listed in tilts[0 .. ntilts).
__global__ void k_flag_tiles(const float* __restrict__ corr, int xb, int yb, int ytiles,
                             const int* __restrict__ tilts, int* __restrict__ tflags) {
  const int tz = tilts ? tilts[blockIdx.z] : (int)blockIdx.z;
  const float* s = corr + (size_t)tz * xb * yb;
  const int ya = blockIdx.y * kApplyTileY, yz = min(yb, ya + kApplyTileY);
  const int half_x = xb / 2;
  const int p0 = half_x * blockIdx.x / kFlagParts, p1 = half_x * (blockIdx.x + 1) / kFlagParts;
  int bad = 0;
#pragma unroll 4  // several rows' loads in flight per thread
  for (int y = ya + threadIdx.y; y < yz; y += blockDim.y) {
    const float2* row = reinterpret_cast<const float2*>(s + (size_t)y * xb);
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
      const float2 v = row[p];
      bad |= (v.x < -1e10f) | (v.y < -1e10f);
    }
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    tflags[((size_t)tz * ytiles + blockIdx.y) * kFlagParts + blockIdx.x] = bad ? 1 : 0;
}

int launch_flag_tiles(Context* c, const float* corr, int xb, int yb, const int* d_tilts,
                      int ntilts, int* tflags, cudaStream_t st) {
  if (ntilts <= 0) return MF_OK;
  const int ytiles = (yb + kApplyTileY - 1) / kApplyTileY;
  dim3 blk(64, 8), grd(kFlagParts, ytiles, ntilts);
  k_flag_tiles<<<grd, blk, 0, st>>>(corr, xb, yb, ytiles, d_tilts, tflags);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// CalcReproj.cu:206-259
void find_proj_range(const float* angles, int nz, const unsigned char* skip, int iproj,
                     int nproj, int* range) {
  const float ref_range = 20.5f, ref_stretch = 1.2f;
  float tilt = angles[iproj];
  float fcos = (float)std::cos(tilt * kD2R);
  int istart = -1;
  for (int i = 0; i < nz; ++i) {
    if (skip[i]) continue;
    float diff = tilt - angles[i];
    if (std::fabs(diff) > ref_range) continue;
    float st = (float)(std::cos(angles[i] * kD2R) / fcos);
    if (st > ref_stretch) continue;
    istart = i;
    break;
  }
  int iend = -1;
  for (int i = (istart < 0 ? 0 : istart); istart >= 0 && i < nz; ++i) {
    if (skip[i]) continue;
    float diff = tilt - angles[i];
    if (std::fabs(diff) > ref_range) continue;
    float st = (float)(std::cos(angles[i] * kD2R) / fcos);
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

// Markerfree/src/method/Util.cpp:8-20
int frame_idx_from_tilt(int nz, const float* a, float tilt) {
  int idx = 0;
  float fmin = (float)std::fabs(tilt - a[0]);
  for (int i = 1; i < nz; ++i) {
    float d = (float)std::fabs(tilt - a[i]);
    if (d >= fmin) continue;
    fmin = d;
    idx = i;
  }
  return idx;
}

// Markerfree/src/method/Util.cpp:22-35
int find_ref_index(int nz, const float* a, int z) {
  int i0 = z - 1, i2 = z + 1;
  if (i0 < 0) i0 = z;
  if (i2 >= nz) i2 = z;
  double t0 = std::fabs(a[i0]), t = std::fabs(a[z]), t2 = std::fabs(a[i2]);
  if (t0 < t) return i0;
  if (t2 < t) return i2;
  return z;
}

}  // namespace mf
