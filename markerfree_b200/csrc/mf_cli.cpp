// Command-line front end with the reference's interface.
//
// Reference: Markerfree/src/main/main.cpp:6-43, opts.h:16-243 (getopt
// "hi:o:n:a:g:m:s:p:", -g O,P,Z,T,A,B,G with exactly seven fields, -s in {0,1},
// -p > 0, -h prints usage and the program then reports wrong input) and
// Process.cpp:34-92 (read, align, write the stack and the parameter file,
// print the elapsed time).  There is no scratch buf.mrc: the stack stays on the
// GPU.
#include <getopt.h>
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/markerfree.h"

namespace {

struct Options {
  char input[255] = "";
  char output[255] = "";
  char initial[255] = "";
  char angle[255] = "";
  float pitch_angle = 0, zshift = 0, offset = 0;
  int thickness = 0, align_z = 600, out_bin = 1, gpu = 0, save_mode = 0, nproj = 10;
  std::string method;
  int iteration = 0;
  float gamma = 0;
  int precision = MF_PREC_FP32;  // --precision (not in the reference)
  bool timing = false;           // --timing (not in the reference): phase times on stderr
};

void usage() {
  std::cout << "[-i INPUT FILENAME]\n    MRC file for reconstruction\n"
            << "[-o OUTPUT FILENAME]\n    MRC filename for result\n"
            << "[-a TILT ANGLE FILENAME]\n    Tilt Angles\n"
            << "[-n INITIAL RECONSTRUCTION]\n    MRC file as initial model (optional)\n"
            << "[-g O,P,Z,T,A,B,G]\n"
            << "    Geometry: offset,pitch_angle,zshift,thickness,AlignZ,OutBin,GPU\n"
            << "[-m METHODS (I,R)]\n    BPT\n    SART: SART iteration_number,relax_parameter\n"
            << "    RP\n"
            << "[-p NPROJ]\n    Number of neighbor projections\n"
            << "[-s SAVE_MODE]\n    SaveParameter (0 or 1)\n"
            << "[--precision fp32|fp16|bf16]\n"
            << "    Re-projection operands (fp32 is the reference's arithmetic)\n"
            << "[--timing]\n    Seconds spent starting the GPU and streaming + aligning\n"
            << "[-h]\n    Help\n";
}

void print_opts(const Options& o) {
  std::cout << "pitch_angle = " << o.pitch_angle << "\n"
            << "zshift = " << o.zshift << "\n"
            << "thickness = " << o.thickness << "\n"
            << "offset = " << o.offset << "\n"
            << "AlignZ = " << o.align_z << "\n"
            << "OutBin = " << o.out_bin << "\n"
            << "GPU = " << o.gpu << "\n"
            << "Savemode = " << o.save_mode << "\n"
            << "nProj = " << o.nproj << "\n"
            << "input = " << o.input << "\n"
            << "output = " << o.output << "\n"
            << "initial = " << o.initial << "\n"
            << "method = " << o.method << "\n"
            << "iter = " << o.iteration << "\n"
            << "step = " << o.gamma << "\n";
}

// opts.h:102-243; returns 1 on success, 0 after -h, -1 on error.
int get_opts(int argc, char** argv, Options* o) {
  static struct option longopts[] = {{"help", no_argument, nullptr, 'h'},
                                     {"input", required_argument, nullptr, 'i'},
                                     {"output", required_argument, nullptr, 'o'},
                                     {"initial", required_argument, nullptr, 'n'},
                                     {"angle", required_argument, nullptr, 'a'},
                                     {"geometry", required_argument, nullptr, 'g'},
                                     {"mode", required_argument, nullptr, 'm'},
                                     {"savemode", required_argument, nullptr, 's'},
                                     {"nproj", required_argument, nullptr, 'p'},
                                     {"precision", required_argument, nullptr, 1000},
                                     {"timing", no_argument, nullptr, 1001},
                                     {nullptr, 0, nullptr, 0}};
  int ch;
  while ((ch = getopt_long(argc, argv, "hi:o:n:a:g:m:s:p:", longopts, nullptr)) != -1) {
    switch (ch) {
      case '?':
        printf("Invalid option '%s'.", argv[optind - 1]);
        fflush(stdout);
        return -1;
      case ':':
        printf("Missing option argument for '%s'.", argv[optind - 1]);
        fflush(stdout);
        return -1;
      case 'h':
        usage();
        return 0;
      case 1001:
        o->timing = true;
        break;
      case 1000:
        if (strcmp(optarg, "fp32") == 0) {
          o->precision = MF_PREC_FP32;
        } else if (strcmp(optarg, "fp16") == 0) {
          o->precision = MF_PREC_FP16;
        } else if (strcmp(optarg, "bf16") == 0) {
          o->precision = MF_PREC_BF16;
        } else {
          printf("precision must be fp32, fp16 or bf16.");
          fflush(stdout);
          return -1;
        }
        break;
      case 'i':
        std::istringstream(optarg) >> o->input;
        break;
      case 'o':
        std::istringstream(optarg) >> o->output;
        break;
      case 'n':
        std::istringstream(optarg) >> o->initial;
        break;
      case 'a':
        std::istringstream(optarg) >> o->angle;
        break;
      case 'g': {
        std::istringstream iss(optarg);
        std::string t;
        if (!std::getline(iss, t, ',')) return -1;
        o->offset = atof(t.c_str());
        if (!std::getline(iss, t, ',')) return -1;
        o->pitch_angle = atof(t.c_str());
        if (!std::getline(iss, t, ',')) return -1;
        o->zshift = atof(t.c_str());
        if (!std::getline(iss, t, ',')) return -1;
        o->thickness = atoi(t.c_str());
        if (!std::getline(iss, t, ',')) return -1;
        o->align_z = atoi(t.c_str());
        if (!std::getline(iss, t, ',')) return -1;
        o->out_bin = atoi(t.c_str());
        if (!std::getline(iss, t)) return -1;
        o->gpu = atoi(t.c_str());
        break;
      }
      case 's':
        o->save_mode = atoi(optarg);
        if (o->save_mode != 0 && o->save_mode != 1) {
          printf("Savemode must be 0 or 1.");
          fflush(stdout);
          return -1;
        }
        break;
      case 'p':
        o->nproj = atoi(optarg);
        if (o->nproj <= 0) {
          printf("nProj must be > 0.");
          fflush(stdout);
          return -1;
        }
        break;
      case 'm': {
        std::istringstream iss(optarg);
        std::string t;
        if (strcmp(optarg, "BPT") != 0 && strcmp(optarg, "RP") != 0) {
          if (!std::getline(iss, o->method, ',')) return -1;
          if (o->method == "SIRT" || o->method == "SART") {
            if (!std::getline(iss, t, ',')) return -1;
            o->iteration = atoi(t.c_str());
            if (!std::getline(iss, t)) return -1;
            o->gamma = atof(t.c_str());
          }
        } else {
          o->method = optarg;
        }
        break;
      }
      default:
        return -1;
    }
  }
  return 1;
}

// Process::DoIt (Process.cpp:34-92)
double now_s() {
  struct timeval t;
  gettimeofday(&t, nullptr);
  return t.tv_sec + t.tv_usec / 1e6;
}

void run(const Options& o) {
  struct timeval t0, t1;
  gettimeofday(&t0, nullptr);
  double tp = now_s();
  auto phase = [&](const char* name) {  // --timing: seconds since the previous phase
    const double t = now_s();
    if (o.timing) fprintf(stderr, "[timing] %s %.3f s\n", name, t - tp);
    tp = t;
  };
  int nx, ny, nz, mode;
  if (mf_mrc_info(o.input, &nx, &ny, &nz, &mode) != MF_OK) {
    printf("[Error] Cannot open input file: %s\n", o.input);
    printf("[Abort] Input stack loading failed. Please check the file path.\n");
    printf("[Abort] DoIt() stopped due to input file loading failure.\n");
    return;
  }
  int na = 0;
  if (mf_read_angles(o.angle, nullptr, 0, &na) != MF_OK) {
    printf("[Error] Cannot open angle file: %s\n", o.angle);
    printf("[Abort] DoIt() stopped due to angle file loading failure.\n");
    return;
  }
  if (na < nz) {
    printf("[Error] Angle file %s holds %d angles for %d images\n", o.angle, na, nz);
    printf("[Abort] DoIt() stopped due to angle file loading failure.\n");
    return;
  }
  std::vector<float> angles(na);
  mf_read_angles(o.angle, angles.data(), na, &na);
  angles.resize(nz);
  phase("header+angles");
  mf_context* ctx = nullptr;
  if (mf_context_create(o.gpu, &ctx) != MF_OK) {
    printf("[Error] %s\n", mf_last_error());
    return;
  }
  phase("gpu-init");
  mf_options mo;
  mo.offset = o.offset;
  mo.pitch_angle = o.pitch_angle;
  mo.zshift = o.zshift;
  mo.thickness = o.thickness;
  mo.align_z = o.align_z;
  mo.out_bin = o.out_bin;
  mo.gpu = o.gpu;
  mo.nproj = o.nproj;
  mo.save_mode = o.save_mode;
  mo.precision = o.precision;
  std::vector<float> sx(nz), sy(nz), rot(nz);
  mf_align_param p{sx.data(), sy.data(), rot.data(), 0.0f};
  int passes = 0;
  // the stack streams from the input file to the GPU and the aligned stack back to
  // the output file (reading, copies and writing overlapped)
  int rc = mf_align_file(ctx, o.input, angles.data(), &mo, &p, o.output, &passes);
  phase("read-align-write");
  mf_context_destroy(ctx);
  if (rc != MF_OK) {
    printf("[Error] alignment failed: %s\n", mf_last_error());
    return;
  }
  gettimeofday(&t1, nullptr);
  double elapsed = (t1.tv_sec - t0.tv_sec) + (t1.tv_usec - t0.tv_usec) / 1e6;
  if (o.align_z != 0) {
    if (mf_save_param(o.output, o.save_mode, &p, angles.data(), nz, nx, ny, o.out_bin,
                      (float)elapsed) != MF_OK) {
      printf("%s\nAlignment data will not be saved\n\n", mf_last_error());
    }
  }
  std::cout << "Elapsed time: " << elapsed << " seconds" << std::endl;
}

}  // namespace

int main(int argc, char* argv[]) {
  Options o;
  if (get_opts(argc, argv, &o) <= 0) {
    printf("***WRONG INPUT.\n");
    fflush(stdout);
    return -1;
  }
  print_opts(o);
  run(o);
  return 0;
}
