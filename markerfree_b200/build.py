"""Build the CUDA library (libmfalign.so) and the command-line tool in-tree.

All device code is compiled for sm_100a only.  Outputs go to markerfree_b200/_build/:
    libmfalign.so   the C-ABI library declared in include/markerfree.h
    Markerfree      the command-line program with the reference's options
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libmfalign.so")
CLI = os.path.join(OUT, "Markerfree")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# deleting an object whose type the file cannot see skips its destructor: an error
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler",
          "-fPIC,-fvisibility=hidden,-Werror=delete-incomplete",
          "-I" + os.path.join(ROOT, "include")] + ARCH
if os.environ.get("MF_HOST_DEBUG"):  # host debug information (backtraces, addr2line)
    CFLAGS += ["-Xcompiler", "-g"]
LIB_SOURCES = ["mf_common.cpp", "mf_io.cpp", "mf_capi.cpp", "mf_correct.cu", "mf_reproj.cu",
               "mf_reproj_tc.cu", "mf_xcorr.cu", "mf_axis.cu", "mf_series.cu", "mf_batch.cu", "mf_serve.cpp",
               "mf_noalloc.cu"]
HEADERS = ["mf_internal.hpp", "mf_xcorr.hpp", "mf_series.hpp"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "markerfree.h")]
    if not _stale(obj, deps):
        return obj
    cmd = [NVCC] + CFLAGS + ["-x", "cu", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, LIB_SOURCES))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-lcufft", "-Xlinker", "-rpath=/usr/local/cuda/lib64"]
        subprocess.run(cmd, check=True)
    cli_src = os.path.join(CSRC, "mf_cli.cpp")
    if _stale(CLI, [cli_src, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), cli_src,
               "-o", CLI, "-L" + OUT, "-lmfalign", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    if verbose:
        print("built", LIB, "and", CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
