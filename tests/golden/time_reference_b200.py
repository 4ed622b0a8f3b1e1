"""Wall time of the reference program and of this library's drop-in program on the
same series file, on the same GPU.

Measurement helper, not a test.  It needs the reference binary built by
oracle/ref/build_ref.sh (oracle/_ref/Markerfree), this repository's build
(markerfree_b200/_build/Markerfree) and one GPU.  It writes the 2048 x 2048 x 61
tilt series (+-60 degrees in 2-degree steps, 300-px slab, seeded phantom) as an
MRC (mode 2) + .rawtlt, then times RUNS runs of each program (this library's
after one untimed run that loads its kernels) with the same command-line options:

    -g 0.0001,0,0,0,300,1,0 -p 10 -s 0

(a non-zero angle offset, so the reference's offset search, which reduces with a
__syncthreads() inside a divergent branch, never runs).  Both programs read the
MRC, align and write the aligned stack and the parameter file; the wall time of
each process is the series time including its file input and output (this
library's program also prints the split: read, GPU start-up, align, write).  Prints
one JSON line with both times, the numbers of projection-matching passes and
final tilt axes each printed, and the parameter differences.

usage: python tests/golden/time_reference_b200.py OUTDIR [RUNS] [SCALE] [REF_TIMEOUT_S]
(REF_TIMEOUT_S <= 0 times this library's program only)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from markerfree_b200 import synth  # noqa: E402
from make_reference_golden import parse_txt, write_mrc  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "Markerfree")
OUR_BIN = os.path.join(ROOT, "markerfree_b200", "_build", "Markerfree")


def run(cmd, log, timeout):
    t0 = time.perf_counter()
    with open(log, "w") as fh:
        rc = subprocess.call(cmd, stdout=fh, stderr=subprocess.STDOUT, timeout=timeout)
    return rc, time.perf_counter() - t0


def passes_and_axis(log):
    txt = open(log, errors="replace").read()
    passes = len(re.findall(r"^f(?:Last)?Err", txt, re.M))
    axes = re.findall(r"New tilt axis:\s+(\S+)", txt)
    return passes, (float(axes[-1]) if axes else None)


def main():
    outdir = sys.argv[1]
    runs = int(sys.argv[2]) if len(sys.argv) > 2 else 2
    scale = float(sys.argv[3]) if len(sys.argv) > 3 else 1.0
    ref_timeout = float(sys.argv[4]) if len(sys.argv) > 4 else 1800.0
    os.makedirs(outdir, exist_ok=True)
    s = synth.config(2, scale=scale)
    mrc = os.path.join(outdir, "series.mrc")
    tlt = os.path.join(outdir, "series.rawtlt")
    write_mrc(mrc, s.stack)
    with open(tlt, "w") as fh:
        for a in s.angles:
            fh.write(f"{a:.2f}\n")
    flags = ["-a", tlt, "-g", f"0.0001,0,0,0,{s.thickness},1,0", "-p", "10", "-s", "0"]
    res = {"series": f"{s.stack.shape[2]}x{s.stack.shape[1]}x{s.stack.shape[0]}",
           "flags": " ".join(flags[2:]), "runs": runs}
    programs = [("reference", REF_BIN, ref_timeout, 0), ("ours", OUR_BIN, 600.0, 1)]
    if ref_timeout <= 0:
        programs = programs[1:]
    for name, binary, tmo, warm in programs:
        out = os.path.join(outdir, f"{name}.mrc")
        # this library's program also reports its phases (--timing, on stderr)
        cmd = [binary, "-i", mrc, "-o", out] + flags + (["--timing"] if name == "ours" else [])
        times = []
        for k in range(runs + warm):
            log = os.path.join(outdir, f"{name}_{k}.log")
            try:
                rc, wall = run(cmd, log, tmo)
            except subprocess.TimeoutExpired:
                rc, wall = "timeout", tmo
            if rc != 0:
                res[name] = {"rc": rc, "log": log}
                break
            if k >= warm:
                times.append(wall)
        else:
            passes, axis = passes_and_axis(os.path.join(outdir, f"{name}_{warm}.log"))
            res[name] = {"wall_s": times, "median_s": float(np.median(times)),
                         "series_per_min": 60.0 / float(np.median(times)),
                         "passes_printed": passes, "final_axis": axis}
            txt = open(os.path.join(outdir, f"{name}_{warm}.log"), errors="replace").read()
            phases = re.findall(r"\[timing\] (\S+) ([0-9.]+) s", txt)
            if phases:
                res[name]["phases_s"] = {k: float(v) for k, v in phases}
            p = parse_txt(out.replace(".mrc", ".txt"))
            res[name + "_params"] = p
        if os.path.exists(out):
            os.remove(out)
    if "reference_params" in res and "ours_params" in res:
        a = np.array(res.pop("reference_params"), np.float64)
        b = np.array(res.pop("ours_params"), np.float64)
        res["d_axis_deg"] = float(np.abs(a[:, 1] - b[:, 1]).max())
        res["d_shift_px"] = float(np.abs(a[:, 2:4] - b[:, 2:4]).max())
    res.pop("reference_params", None)
    res.pop("ours_params", None)
    os.remove(mrc)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
