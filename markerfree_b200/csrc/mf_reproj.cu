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

// ---------------------------------------------------------------------------
// Device geometry helpers.  Every step is an explicitly rounded IEEE operation so
// that no multiply-add is contracted: cell and bin indices then agree bit for bit
// with a plain C evaluation of the reference expressions.
struct RayStart {
  float tx, tz, zst;
};

__device__ __forceinline__ RayStart ray_start(int bx, int xb, int W, int T, float fcos,
                                              float fsin, int L) {
  float fxp = __fsub_rn(__fadd_rn((float)bx, 0.5f), __fmul_rn((float)xb, 0.5f));
  RayStart r;
  r.tx = __fadd_rn(__fmul_rn(fxp, fcos), __fmul_rn((float)W, 0.5f));
  r.tz = __fadd_rn(__fmul_rn(fxp, fsin), __fmul_rn((float)T, 0.5f));
  r.zst = __fsub_rn(__fdiv_rn(__fmul_rn(-fxp, fsin), fcos), __fmul_rn(0.5f, (float)L));
  return r;
}

// Sample j of a ray; returns false when outside [0, W-1) x [0, T-1).
__device__ __forceinline__ bool ray_cell(const RayStart& r, int j, int W, int T, float fcos,
                                         float fsin, int* ix, int* iz) {
  float fz = __fadd_rn((float)j, r.zst);
  float X = __fsub_rn(r.tx, __fmul_rn(fz, fsin));
  float Z = __fadd_rn(r.tz, __fmul_rn(fz, fcos));
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
  float v = __fadd_rn(__fadd_rn(__fmul_rn(fx, c), __fmul_rn(fz, s)), cent);
  if (v < 0.0f || v > (float)(xb - 1)) return -1;
  return (int)v;
}

// ---------------------------------------------------------------------------
// Exact path: one thread per (detector column, row).
__global__ void k_reproject_exact(const float* __restrict__ corr, int xb, int yb, size_t pix,
                                  const float* __restrict__ bp, int i0, int nk, float fcos,
                                  float fsin, int L, int T, const int* __restrict__ rowflags,
                                  float* __restrict__ out) {
  int bx = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (bx >= xb || y >= yb) return;
  if (rowflags && rowflags[y / kApplyTileY] == 0) return;
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  RayStart r = ray_start(bx, xb, W, T, fcos, fsin, L);
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
      fint = __fadd_rn(fint, __fmul_rn(__fmul_rn(v, c), w));
      fcount = __fadd_rn(fcount, w);
    }
    float cell = (fcount < 0.001f) ? kSentinel : __fdiv_rn(fint, fcount);
    if (cell >= -1e10f) {
      sum = __fadd_rn(sum, cell);
      cnt += 1;
    }
  }
  float res = ((float)cnt < __fmul_rn(0.8f, (float)L)) ? kSentinel : __fdiv_rn(sum, (float)cnt);
  out[(size_t)y * xb + bx] = res;
}

int launch_reproject_exact(Context* c, const float* corr, int xb, int yb, size_t pix,
                           const float* d_bp, int i0, int nk, float fcos, float fsin, int ray_len,
                           int thick, const int* d_rowflags, float* out, cudaStream_t st) {
  dim3 blk(128, 1), grd((xb + 127) / 128, yb);
  k_reproject_exact<<<grd, blk, 0, st>>>(corr, xb, yb, pix, d_bp, i0, nk, fcos, fsin, ray_len,
                                         thick, d_rowflags, out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Operator build, pass 1: per column the number of valid ray samples and, per
// neighbour, the range of sinogram bins touched.
__global__ void k_op_scan(int xb, int T, const float* __restrict__ bp, int nk, float fcos,
                          float fsin, int L, int* __restrict__ cnt, int* __restrict__ lo,
                          int* __restrict__ hi) {
  int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= xb) return;
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  RayStart r = ray_start(bx, xb, W, T, fcos, fsin, L);
  int n = 0;
  for (int k = 0; k < nk; ++k) {
    lo[bx * nk + k] = INT_MAX;
    hi[bx * nk + k] = -1;
  }
  for (int j = 0; j < L; ++j) {
    int ix, iz;
    if (!ray_cell(r, j, W, T, fcos, fsin, &ix, &iz)) continue;
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
      if (b < lo[bx * nk + k]) lo[bx * nk + k] = b;
      if (b > hi[bx * nk + k]) hi[bx * nk + k] = b;
    }
  }
  cnt[bx] = n;
}

// Pass 2: accumulate coefficients.  seg[t*nk + k] = (row offset within the tile,
// first bin).  Each thread owns one column of its tile, so there are no races.
__global__ void k_op_fill(int xb, int T, const float* __restrict__ bp, int nk, float fcos,
                          float fsin, int L, const int* __restrict__ cnt,
                          const OpTile* __restrict__ tiles, const int2* __restrict__ seg,
                          float* __restrict__ coef, int* __restrict__ colvalid) {
  int bx = blockIdx.x * blockDim.x + threadIdx.x;
  if (bx >= xb) return;
  const int n = cnt[bx];
  const bool valid = !((float)n < __fmul_rn(0.8f, (float)L));
  colvalid[bx] = valid ? 1 : 0;
  if (!valid) return;
  const int W = 2 * xb;
  const float cent = __fmul_rn((float)xb, 0.5f);
  const int t = bx / kOpTileX, xl = bx % kOpTileX;
  const OpTile tile = tiles[t];
  const float inv_n = 1.0f / (float)n;
  RayStart r = ray_start(bx, xb, W, T, fcos, fsin, L);
  for (int j = 0; j < L; ++j) {
    int ix, iz;
    if (!ray_cell(r, j, W, T, fcos, fsin, &ix, &iz)) continue;
    float fcount = 0.0f;
    for (int k = 0; k < nk; ++k) {
      int b = cell_bin(ix, iz, W, T, bp[3 * k + 1], bp[3 * k + 2], cent, xb);
      if (b >= 0) fcount = __fadd_rn(fcount, bp[3 * k]);
    }
    if (fcount < 0.001f) continue;
    for (int k = 0; k < nk; ++k) {
      int b = cell_bin(ix, iz, W, T, bp[3 * k + 1], bp[3 * k + 2], cent, xb);
      if (b < 0) continue;
      int2 sg = seg[t * nk + k];
      size_t row = (size_t)tile.row0 + sg.x + (b - sg.y);
      float term = bp[3 * k + 1] * bp[3 * k] / fcount * inv_n;
      coef[row * kOpTileX + xl] += term;
    }
  }
}

int build_reproj_op(Context* c, const ReprojGeom& g, ReprojOp* op, cudaStream_t st) {
  const int xb = g.xb, nk = g.nk;
  DevBuf d_bp, d_cnt, d_lo, d_hi;
  MF_TRY(d_bp.alloc(sizeof(float) * g.bp.size()));
  MF_TRY(d_cnt.alloc(sizeof(int) * xb));
  MF_TRY(d_lo.alloc(sizeof(int) * xb * nk));
  MF_TRY(d_hi.alloc(sizeof(int) * xb * nk));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_bp.p, g.bp.data(), sizeof(float) * g.bp.size(),
                                cudaMemcpyHostToDevice, st));
  k_op_scan<<<(xb + 127) / 128, 128, 0, st>>>(xb, g.thick, d_bp.as<float>(), nk, g.fcos, g.fsin,
                                              g.ray_len, d_cnt.as<int>(), d_lo.as<int>(),
                                              d_hi.as<int>());
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  std::vector<int> lo((size_t)xb * nk), hi((size_t)xb * nk);
  MF_CHECK_CUDA(cudaMemcpyAsync(lo.data(), d_lo.p, sizeof(int) * lo.size(),
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(hi.data(), d_hi.p, sizeof(int) * hi.size(),
                                cudaMemcpyDeviceToHost, st));
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  // Tile layout.
  const int ntiles = (xb + kOpTileX - 1) / kOpTileX;
  std::vector<OpTile> tiles(ntiles);
  std::vector<int2> seg((size_t)ntiles * nk);
  std::vector<int2> rowmap;
  int total = 0;
  for (int t = 0; t < ntiles; ++t) {
    int x0 = t * kOpTileX, x1 = std::min(xb, x0 + kOpTileX);
    int rows = 0;
    for (int k = 0; k < nk; ++k) {
      int l = INT_MAX, h = -1;
      for (int x = x0; x < x1; ++x) {
        l = std::min(l, lo[(size_t)x * nk + k]);
        h = std::max(h, hi[(size_t)x * nk + k]);
      }
      if (h < 0) {
        seg[(size_t)t * nk + k] = make_int2(rows, 0);
        continue;
      }
      seg[(size_t)t * nk + k] = make_int2(rows, l);
      for (int b = l; b <= h; ++b) rowmap.push_back(make_int2(g.i0 + k, b));
      rows += h - l + 1;
    }
    int padded = (rows + kOpChunk - 1) / kOpChunk * kOpChunk;
    if (padded == 0) padded = kOpChunk;
    for (int r = rows; r < padded; ++r) rowmap.push_back(make_int2(g.i0, 0));
    tiles[t].row0 = total;
    tiles[t].rows = padded;
    total += padded;
  }
  op->ip = g.ip;
  op->i0 = g.i0;
  op->i1 = g.i1;
  op->xb = xb;
  op->yb = g.yb;
  op->thick = g.thick;
  op->ray_len = g.ray_len;
  op->ntiles = ntiles;
  op->total_rows = total;
  MF_TRY(op->coef.alloc(sizeof(float) * (size_t)total * kOpTileX));
  MF_TRY(op->rowmap.alloc(sizeof(int2) * (size_t)total));
  MF_TRY(op->tiles.alloc(sizeof(OpTile) * ntiles));
  MF_TRY(op->colvalid.alloc(sizeof(int) * xb));
  DevBuf d_seg;
  MF_TRY(d_seg.alloc(sizeof(int2) * seg.size()));
  MF_CHECK_CUDA(cudaMemsetAsync(op->coef.p, 0, sizeof(float) * (size_t)total * kOpTileX, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(op->rowmap.p, rowmap.data(), sizeof(int2) * rowmap.size(),
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(op->tiles.p, tiles.data(), sizeof(OpTile) * ntiles,
                                cudaMemcpyHostToDevice, st));
  MF_CHECK_CUDA(cudaMemcpyAsync(d_seg.p, seg.data(), sizeof(int2) * seg.size(),
                                cudaMemcpyHostToDevice, st));
  k_op_fill<<<(xb + 127) / 128, 128, 0, st>>>(xb, g.thick, d_bp.as<float>(), nk, g.fcos, g.fsin,
                                              g.ray_len, d_cnt.as<int>(), op->tiles.as<OpTile>(),
                                              d_seg.as<int2>(), op->coef.as<float>(),
                                              op->colvalid.as<int>());
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  // the temporaries are freed when this returns; wait for the kernels using them
  MF_CHECK_CUDA(cudaStreamSynchronize(st));
  return MF_OK;
}

// ---------------------------------------------------------------------------
// Operator apply: out[y][x] = sum_r A[y][r] * B_t[r][x] with A gathered from the
// neighbour rows through rowmap.  64 x 64 output tile per CTA, 256 threads with
// a 4 x 4 register micro-tile each.
__global__ void __launch_bounds__(256) k_op_apply(const float* __restrict__ corr, int xb, int yb,
                                                  size_t pix, const float* __restrict__ coef,
                                                  const int2* __restrict__ rowmap,
                                                  const OpTile* __restrict__ tiles,
                                                  const int* __restrict__ colvalid,
                                                  int* __restrict__ rowflags,
                                                  float* __restrict__ out) {
  __shared__ __align__(16) float As[kOpChunk][kApplyTileY];
  __shared__ __align__(16) float Bs[kOpChunk][kOpTileX];
  __shared__ int s_flag;
  const int t = blockIdx.x;
  const int y0 = blockIdx.y * kApplyTileY;
  const int x0 = t * kOpTileX;
  const OpTile tile = tiles[t];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  if (tid == 0) s_flag = 0;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  const int lr = tid % kOpChunk;  // operator row this thread loads for A
  const int ly = tid / kOpChunk;  // base row of y
  bool bad = false;
  __syncthreads();
  for (int r0 = 0; r0 < tile.rows; r0 += kOpChunk) {
    const int row = tile.row0 + r0;
    int2 rm = rowmap[row + lr];
    const float* src = corr + (size_t)rm.x * pix + rm.y;
#pragma unroll
    for (int q = 0; q < kApplyTileY / 16; ++q) {
      int yy = ly + 16 * q;
      int y = y0 + yy;
      float v = 0.0f;
      if (y < yb) {
        v = __ldg(src + (size_t)y * xb);
        bad |= (v < -1e10f);
      }
      As[lr][yy] = v;
    }
    const float4* cb = reinterpret_cast<const float4*>(coef + (size_t)row * kOpTileX);
    reinterpret_cast<float4*>(&Bs[0][0])[tid] = __ldg(cb + tid);
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < kOpChunk; ++rr) {
      float4 a = *reinterpret_cast<const float4*>(&As[rr][ty * 4]);
      float4 b = *reinterpret_cast<const float4*>(&Bs[rr][tx * 4]);
      float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();
  }
  if (bad) s_flag = 1;
  __syncthreads();
  if (tid == 0 && s_flag) atomicOr(&rowflags[blockIdx.y], 1);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int y = y0 + ty * 4 + i;
    if (y >= yb) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int x = x0 + tx * 4 + j;
      if (x >= xb) continue;
      out[(size_t)y * xb + x] = colvalid[x] ? acc[i][j] : kSentinel;
    }
  }
}

int launch_reproject_apply(Context* c, const ReprojOp& op, const float* corr, size_t pix,
                           int* d_rowflags, float* out, cudaStream_t st) {
  dim3 grd(op.ntiles, (op.yb + kApplyTileY - 1) / kApplyTileY);
  k_op_apply<<<grd, 256, 0, st>>>(corr, op.xb, op.yb, pix, op.coef.as<float>(),
                                  op.rowmap.as<int2>(), op.tiles.as<OpTile>(),
                                  op.colvalid.as<int>(), d_rowflags, out);
  c->launches++;
  MF_CHECK_CUDA(cudaGetLastError());
  return MF_OK;
}

// ---------------------------------------------------------------------------
// CalcReproj.cu:281-334
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
