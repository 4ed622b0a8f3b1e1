/* Single-process stand-in for the MPI subset the reference program uses.
 *
 * TEST INFRASTRUCTURE ONLY.  It lets the unmodified reference sources build into
 * oracle/_ref/ so that the reference can be run on one GPU to produce its own
 * outputs for parity checks.  The reference uses MPI only for start-up, two
 * broadcasts from rank 0 and file I/O (Markerfree/src/main/main.cpp:8-11,40-41,
 * Markerfree/src/main/Process.cpp:144,156, Markerfree/src/mrc/mrcstack.cpp), so
 * with one rank every call maps to stdio.
 */
#ifndef MF_REF_MPI_SHIM_H
#define MF_REF_MPI_SHIM_H

#include <stdio.h>
#include <string.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef FILE* MPI_File;
typedef struct { int unused; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_FILE_NULL ((MPI_File)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_CREATE 1
#define MPI_SEEK_SET SEEK_SET
#define MPI_SEEK_CUR SEEK_CUR

static inline int mf_shim_type_size(MPI_Datatype t) { return t == MPI_CHAR ? 1 : 4; }

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Get_processor_name(char* name, int* len) {
  strcpy(name, "localhost");
  *len = (int)strlen(name);
  return 0;
}
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c;
  return 0;
}
static inline int MPI_Error_string(int code, char* s, int* len) {
  snprintf(s, MPI_MAX_ERROR_STRING, "I/O error %d", code);
  *len = (int)strlen(s);
  return 0;
}
static inline int MPI_File_open(MPI_Comm c, const char* name, int mode, MPI_Info info,
                                MPI_File* fh) {
  (void)c; (void)info;
  FILE* f = 0;
  if (mode & MPI_MODE_RDONLY) {
    f = fopen(name, "rb");
  } else {
    f = fopen(name, "r+b");
    if (!f && (mode & MPI_MODE_CREATE)) f = fopen(name, "w+b");
  }
  *fh = f;
  return f ? 0 : 1;
}
static inline int MPI_File_close(MPI_File* fh) {
  if (*fh) fclose(*fh);
  *fh = 0;
  return 0;
}
static inline int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
  if (!fh) return 1;
  fflush(fh);
  return ftruncate(fileno(fh), (off_t)size) == 0 ? 0 : 1;
}
static inline int MPI_File_seek(MPI_File fh, MPI_Offset off, int whence) {
  if (!fh) return 1;
  return fseeko(fh, (off_t)off, whence) == 0 ? 0 : 1;
}
static inline int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype t,
                                MPI_Status* st) {
  (void)st;
  if (!fh) return 1;
  size_t want = (size_t)count * (size_t)mf_shim_type_size(t);
  return fread(buf, 1, want, fh) == want ? 0 : 1;
}
static inline int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype t,
                                 MPI_Status* st) {
  (void)st;
  if (!fh) return 1;
  size_t want = (size_t)count * (size_t)mf_shim_type_size(t);
  return fwrite(buf, 1, want, fh) == want ? 0 : 1;
}

#endif
