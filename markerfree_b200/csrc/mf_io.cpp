// File formats: MRC stacks, .rawtlt angles, .txt / .xf parameter files.
//
// Reference: Markerfree/src/mrc/mrcheader.h:24-96 (1024-byte header),
// mrcstack.cpp:51-119 (modes 0/1/2, extended header skipped), :421-501
// (InitializeHeader + UpdateHeader for the float output), Process.cpp:186-206
// (angles), SaveParam.cpp:15-262 (.xf and .txt writers).  The reference does all
// of this through MPI-IO; a single process needs plain stdio.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "mf_internal.hpp"

using mf::set_error;

namespace {

#pragma pack(push, 1)
struct MrcHeader {
  int nx, ny, nz, mode;
  int nxstart, nystart, nzstart;
  int mx, my, mz;
  float xlen, ylen, zlen;
  float alpha, beta, gamma;
  int mapc, mapr, maps;
  float amin, amax, amean;
  short ispg, nsymbt;
  int next;
  short creatid;
  char blank[30];
  short nint, nreal, sub, zfac;
  float min2, max2, min3, max3, min4, max4;
  short idtype, lens, nd1, nd2, vd1, vd2;
  float tiltangles[6];
  float xorg, yorg, zorg;
  char cmap[4];
  char stamp[4];
  float rms;
  int nlabl;
  char labels[10][80];
};
#pragma pack(pop)
static_assert(sizeof(MrcHeader) == 1024, "MRC header must be 1024 bytes");

int read_header(FILE* f, MrcHeader* h) {
  if (fread(h, 1, sizeof(*h), f) != sizeof(*h)) return set_error(MF_ERR_FORMAT, "short MRC header");
  if (h->nx <= 0 || h->ny <= 0 || h->nz <= 0)
    return set_error(MF_ERR_FORMAT, "invalid MRC dimensions %d x %d x %d", h->nx, h->ny, h->nz);
  if (h->mode != 0 && h->mode != 1 && h->mode != 2)
    return set_error(MF_ERR_FORMAT, "File type unknown! (MRC mode %d)", h->mode);
  if (h->next < 0) return set_error(MF_ERR_FORMAT, "negative extended header size");
  return MF_OK;
}

}  // namespace

extern "C" {

MF_API int mf_mrc_info(const char* path, int* nx, int* ny, int* nz, int* mode) {
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MF_ERR_IO, "Cannot open input file: %s", path);
  MrcHeader h;
  int rc = read_header(f, &h);
  fclose(f);
  if (rc != MF_OK) return rc;
  if (nx) *nx = h.nx;
  if (ny) *ny = h.ny;
  if (nz) *nz = h.nz;
  if (mode) *mode = h.mode;
  return MF_OK;
}

MF_API int mf_mrc_read(const char* path, float* out) {
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MF_ERR_IO, "Cannot open input file: %s", path);
  MrcHeader h;
  int rc = read_header(f, &h);
  if (rc != MF_OK) {
    fclose(f);
    return rc;
  }
  size_t pix = (size_t)h.nx * h.ny;
  size_t psize = h.mode == 0 ? 1 : (h.mode == 1 ? 2 : 4);
  if (fseeko(f, (off_t)sizeof(MrcHeader) + h.next, SEEK_SET) != 0) {
    fclose(f);
    return set_error(MF_ERR_IO, "seek failed in %s", path);
  }
  std::vector<unsigned char> buf(pix * psize);
  for (int z = 0; z < h.nz; ++z) {
    if (fread(buf.data(), 1, buf.size(), f) != buf.size()) {
      fclose(f);
      return set_error(MF_ERR_FORMAT, "MRC file %s is truncated at slice %d", path, z);
    }
    float* o = out + (size_t)z * pix;
    if (h.mode == 0) {
      for (size_t i = 0; i < pix; ++i) o[i] = (float)buf[i];
    } else if (h.mode == 1) {
      const short* s = reinterpret_cast<const short*>(buf.data());
      for (size_t i = 0; i < pix; ++i) o[i] = (float)s[i];
    } else {
      memcpy(o, buf.data(), pix * 4);
    }
  }
  fclose(f);
  return MF_OK;
}

}  // extern "C"

namespace mf {

// The float32 output header: InitializeHeader + SetSize + UpdateHeader.
void mrc_float_header(const float* mid, int nx, int ny, int nz, void* out1024) {
  MrcHeader h;
  memset(&h, 0, sizeof(h));
  // InitializeHeader + SetSize (mrcstack.cpp:421-454, mrcstack.h:170-175)
  h.mode = 2;
  h.mx = nx;
  h.my = ny;
  h.mz = nz;
  h.xlen = h.ylen = h.zlen = 1;
  h.alpha = h.beta = h.gamma = 90;
  h.mapc = 1;
  h.mapr = 2;
  h.maps = 3;
  h.creatid = 1000;
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  // UpdateHeader (mrcstack.cpp:456-501): statistics of the middle slice only,
  // amax starting from FLT_MIN, sentinels skipped.
  size_t pix = (size_t)nx * ny;
  float amin = FLT_MAX, amax = FLT_MIN;
  long double amean = 0;
  int count = 0;
  for (size_t i = pix; i--;) {
    float v = mid[i];
    if (v < (float)-1e10) continue;
    if (v > amax) amax = v;
    if (v < amin) amin = v;
    amean += v;
    count++;
  }
  amean /= count;
  h.amin = amin;
  h.amax = amax;
  h.amean = (float)amean;
  h.nlabl = 0;
  memcpy(out1024, &h, sizeof(h));
}

// Open an MRC stack for reading, positioned at its first data byte.
int mrc_open_stack(const char* path, FILE** fp, int* nx, int* ny, int* nz, int* mode) {
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MF_ERR_IO, "Cannot open input file: %s", path);
  MrcHeader h;
  int rc = read_header(f, &h);
  if (rc == MF_OK && fseeko(f, (off_t)sizeof(MrcHeader) + h.next, SEEK_SET) != 0)
    rc = set_error(MF_ERR_IO, "seek failed in %s", path);
  if (rc != MF_OK) {
    fclose(f);
    return rc;
  }
  *fp = f;
  *nx = h.nx;
  *ny = h.ny;
  *nz = h.nz;
  *mode = h.mode;
  return MF_OK;
}

}  // namespace mf

extern "C" {

MF_API int mf_mrc_write(const char* path, const float* data, int nx, int ny, int nz) {
  if (!path || !data || nx <= 0 || ny <= 0 || nz <= 0) return set_error(MF_ERR_ARG, "invalid MRC write");
  const size_t pix = (size_t)nx * ny;
  unsigned char h[1024];
  mf::mrc_float_header(data + (size_t)(int)(nz * .5) * pix, nx, ny, nz, h);
  FILE* f = fopen(path, "wb");
  if (!f) return set_error(MF_ERR_IO, "cannot open %s for writing", path);
  bool ok = fwrite(h, 1, sizeof(h), f) == sizeof(h);
  ok = ok && fwrite(data, sizeof(float), pix * nz, f) == pix * nz;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return set_error(MF_ERR_IO, "write failed on %s", path);
  return MF_OK;
}

MF_API int mf_read_angles(const char* path, float* out, int max, int* n) {
  std::ifstream in(path);
  if (!in.good()) return set_error(MF_ERR_IO, "Cannot open angle file: %s", path);
  int k = 0;
  while (in.good()) {
    float v;
    in >> v;
    if (in.fail()) break;
    if (out && k < max) out[k] = v;
    k++;
  }
  if (n) *n = k;
  return MF_OK;
}

MF_API int mf_save_param(const char* output_path, int mode, const mf_align_param* p,
                         const float* file_angles, int nz, int raw_nx, int raw_ny, int out_bin,
                         float elapsed_s) {
  if (!output_path || !p || !file_angles || nz < 1) return set_error(MF_ERR_ARG, "invalid argument");
  if (mode != 0 && mode != 1) return set_error(MF_ERR_ARG, "Savemode must be 0 or 1.");
  // CollectParam (Process.cpp:399-418): angles as read, ascending; inv when reversed
  std::vector<float> angles(file_angles, file_angles + nz);
  bool inv = false;
  if (nz > 1 && angles[0] > angles[1]) {
    std::vector<float> r(angles.rbegin(), angles.rend());
    angles.swap(r);
    inv = true;
  }
  char filename[4096];
  snprintf(filename, sizeof(filename), "%s", output_path);
  char* pc = strstr(filename, ".mrc");
  const char* ext = mode == 0 ? ".txt" : ".xf";
  if (pc)
    strcpy(pc, ext);
  else
    strncat(filename, ext, sizeof(filename) - strlen(filename) - 1);
  FILE* f = fopen(filename, "wt");
  if (!f) return set_error(MF_ERR_IO, "Unable to open %s.", filename);
  const int mbin = 1;  // GetParam(1, ...) at Process.cpp:416
  if (mode == 0) {
    fprintf(f, "# Markerfree Alignment\n");
    fprintf(f, "# RawSize = %d %d %d\n", raw_nx, raw_ny, nz);
    fprintf(f, "# SEC       ROT          TX        TY         TILT\n");
    for (int i = 0; i < nz; ++i) {
      float sx = p->shift_x[i] * mbin, sy = p->shift_y[i] * mbin;
      fprintf(f, "%5d   %9.4f  %9.3f  %9.3f   %8.2f\n", i, p->rotate[i], sx, sy, angles[i]);
    }
    fprintf(f, "angleoffset: %f\n", p->angle_offset);
    fprintf(f, "Output Bin: %d\n", out_bin);
    fprintf(f, "Elapsed time: %f seconds\n", elapsed_s);
  } else {
    // SaveXf (SaveParam.cpp:15-53); height is taken from X as in the reference
    const float width = (float)raw_nx, height = (float)raw_nx;
    const float cx = width / 2.0f, cy = height / 2.0f;
    int start = inv ? nz - 1 : 0, end = inv ? -1 : nz, step = inv ? -1 : 1;
    for (int i = start; i != end; i += step) {
      float sx = p->shift_x[i] * mbin, sy = p->shift_y[i] * mbin;
      float th = p->rotate[i] * M_PI / 180.0f;
      float c = cos(th), s = sin(th);
      float T1 = -sx - cx + c * cx - s * cy;
      float T2 = -sy - cy + s * cx + c * cy;
      float par[6] = {c, s, -s, c, T1 * c + T2 * s - cx + c * cx + s * cy,
                      -T1 * s + T2 * c - cy - s * cx + c * cy};
      fprintf(f, "%9.3f  %9.3f  %9.3f  %9.3f  %9.3f  %9.3f \n", par[0], par[1], par[2], par[3],
              par[4], par[5]);
    }
  }
  if (fclose(f) != 0) return set_error(MF_ERR_IO, "write failed on %s", filename);
  return MF_OK;
}

}  // extern "C"
