#!/usr/bin/env bash
# Build the unmodified reference program from its own sources into oracle/_ref/.
#
# TEST INFRASTRUCTURE ONLY.  The reference is compiled where it lies (read-only,
# nothing is copied into this repository) with nvcc for sm_100a, linked against
# cuFFT, and given oracle/ref/mpi.h in place of an MPI installation.  The binary
# is used to produce the reference's own outputs on synthetic inputs.
#
# usage: oracle/ref/build_ref.sh [REFERENCE_ROOT]
# (default: $MF_REFERENCE_ROOT, else a checkout named `reference` beside this repository)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF=${1:-${MF_REFERENCE_ROOT:-$HERE/../../../reference}}
SRC="$REF/Markerfree/src"
OUT="$HERE/../_ref"
OBJ="$OUT/obj"
mkdir -p "$OBJ"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
FLAGS=(-O3 -std=c++14 -gencode arch=compute_100a,code=sm_100a -I"$HERE" -I"$SRC"
       -Xcompiler -fopenmp -w)
objs=()
i=0
for f in "$SRC"/main/main.cpp "$SRC"/main/Process.cpp "$SRC"/mrc/mrcstack.cpp \
         "$SRC"/method/*.cpp "$SRC"/method/*.cu; do
  o="$OBJ/$i.o"
  i=$((i + 1))
  if [[ "$f" == *.cu ]]; then
    "$NVCC" "${FLAGS[@]}" -x cu -dc -c "$f" -o "$o"
  else
    "$NVCC" "${FLAGS[@]}" -x cu -dc -c "$f" -o "$o"
  fi
  objs+=("$o")
done
"$NVCC" -gencode arch=compute_100a,code=sm_100a "${objs[@]}" -o "$OUT/Markerfree" \
  -lcufft -lgomp -Xlinker -rpath=/usr/local/cuda/lib64
echo "built $OUT/Markerfree"
