"""Run the reference program on seeded synthetic series and keep its outputs.

Test-fixture generator.  It needs the reference binary built by
oracle/ref/build_ref.sh (oracle/_ref/Markerfree) and one GPU.  For each case it
writes the series as an MRC (mode 2) + .rawtlt, runs the reference with the
case's flags, and stores in OUTDIR/<case>/:
    ref.txt        the reference's parameter file
    ref.log        its stdout (per-pass measured shifts, Z centre, tilt axes)
    aligned.npz    per-slice sum / sum of squares of the aligned stack and a
                   64x64 crop of the middle slice
    case.json      the generator arguments and flags

The tilt-angle offset search of the reference (FindOffset.cu:85-238) reduces with
a __syncthreads() inside a divergent branch (FindOffset.cu:57-65), which CUDA
leaves undefined and which may hang a GPU, so every case passes a non-zero offset
(-g O,... with O = 1e-4 degrees) and the search is never run.

usage: python tests/golden/make_reference_golden.py OUTDIR [case ...]
       python tests/golden/make_reference_golden.py --fixtures OUTDIR [case ...]

The second form turns the run outputs in OUTDIR into the committed fixtures
tests/golden/ref_<case>.json (generator arguments, flags, the events the
reference printed, its final parameters and per-slice sums of its aligned
stack), ref_<case>.txt (its parameter file) and ref_<case>_crop.npy (a 64 x 64
crop of the middle aligned slice).
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

from markerfree_b200 import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "Markerfree")

# A case name ending in "_p<k>" runs the base case with its stack multiplied by
# 1 + 1e-6 * U(-1, 1) (seed k): the spread of the reference's own results over
# such perturbations bounds how closely any other implementation can follow it.
# A name ending in "_s1" runs the base case with -s 1, so the reference writes its
# parameters as an IMOD .xf file (SaveParam.cpp:15-120) instead of the .txt.
# "cfg2" is the realistic single-series configuration (synth.config(2): 2048^2 x 61
# tilts, T = 300, SNR 0.05), generated by the config function rather than kwargs.
CASES = {
    # name: (generator kwargs, thickness, nproj, timeout s)
    "c1s256": (dict(nx=256, ny=256, vol_z=64, n_blobs=80, seed=1101, snr=0.5,
                    shift_sd=3.0), 60, 10, 600),
    "c1s256b": (dict(nx=256, ny=192, vol_z=48, n_blobs=60, seed=1102, snr=0.2,
                     tilt_step=2.0, tilt_min=-50, tilt_max=50, axis=93.0, shift_sd=4.0),
                40, 6, 600),
    "cfg1": (dict(nx=512, ny=512, vol_z=128, n_blobs=200, seed=1001, snr=0.1,
                  shift_sd=4.0), 100, 10, 1200),
    # a well-conditioned series: high SNR, the alignment settles in few passes
    "hi384": (dict(nx=384, ny=384, vol_z=96, n_blobs=160, seed=1201, snr=4.0, shift_sd=3.0,
                   axis=87.0), 80, 10, 1200),
    "cfg2": (dict(config=2), 300, 10, 1800),
    # wide enough that the reference bins the projection matching by 2
    # (ProjAlign.cpp:57-61: round(3072 / 2048) = 2; slab 100 / 2 = 50)
    "bin2": (dict(nx=3072, ny=320, vol_z=64, n_blobs=240, seed=1301, snr=4.0, shift_sd=3.0,
                  axis=87.0, tilt_min=-40, tilt_max=40, tilt_step=4.0), 100, 10, 1200),
}


def case_spec(name):
    """(generator kwargs, thickness, nproj, timeout, perturbation seed or None, save mode)."""
    save = 0
    if name.endswith("_s1"):
        name, save = name[:-3], 1
    base, _, tag = name.partition("_p")
    kw, thick, nproj, tmo = CASES[base]
    return kw, thick, nproj, tmo, (int(tag) if tag else None), save


def make_case_series(kw, thick, nproj):
    """The case's series: synth.config(n) for {"config": n}, else make_series(**kw)."""
    if "config" in kw:
        return synth.config(kw["config"])
    return synth.make_series(thickness=thick, nproj=nproj, **kw)


def perturbed(stack, seed):
    rng = np.random.default_rng(seed)
    return (stack * (1.0 + 1e-6 * rng.uniform(-1.0, 1.0, stack.shape))).astype(np.float32)


def write_mrc(path, stack, mode=2):
    nz, ny, nx = stack.shape
    hdr = np.zeros(256, np.int32)
    hdr[0:4] = [nx, ny, nz, mode]
    hdr[7:10] = [nx, ny, nz]
    f = hdr.view(np.float32)
    f[10:13] = [nx, ny, nz]
    f[13:16] = [90, 90, 90]
    hdr[16:19] = [1, 2, 3]
    data = stack.astype(np.int16 if mode == 1 else np.float32)
    f[19], f[20], f[21] = float(data.min()), float(data.max()), float(data.mean())
    raw = bytearray(hdr.tobytes())
    raw[208:212] = b"MAP "
    raw[212:216] = bytes([0x44, 0x44, 0, 0])
    with open(path, "wb") as fh:
        fh.write(bytes(raw))
        fh.write(data.tobytes())


def read_mrc_float(path):
    with open(path, "rb") as fh:
        hdr = np.frombuffer(fh.read(1024), np.int32)
        nx, ny, nz, mode = (int(v) for v in hdr[:4])
        nxt = int(hdr[23])
        fh.seek(1024 + nxt)
        data = np.frombuffer(fh.read(), np.float32, count=nx * ny * nz)
    return data.reshape(nz, ny, nx)


def run_case(outdir, name):
    kw, thick, nproj, tmo, pert, save = case_spec(name)
    s = make_case_series(kw, thick, nproj)
    d = os.path.join(outdir, name)
    os.makedirs(d, exist_ok=True)
    mrc = os.path.join(d, "in.mrc")
    tlt = os.path.join(d, "in.rawtlt")
    write_mrc(mrc, s.stack if pert is None else perturbed(s.stack, pert))
    with open(tlt, "w") as fh:
        for a in s.angles:
            fh.write(f"{a:.2f}\n")
    out = os.path.join(d, "out.mrc")
    cmd = [REF_BIN, "-i", mrc, "-o", out, "-a", tlt, "-g", f"0.0001,0,0,0,{thick},1,0",
           "-p", str(nproj), "-s", str(save)]
    t0 = time.time()
    with open(os.path.join(d, "ref.log"), "w") as log:
        rc = subprocess.call(cmd, stdout=log, stderr=subprocess.STDOUT, timeout=tmo)
    wall = time.time() - t0
    if rc == 0 and os.path.exists(out):
        al = read_mrc_float(out)
        mid = al.shape[0] // 2
        cy, cx = al.shape[1] // 2, al.shape[2] // 2
        np.savez_compressed(os.path.join(d, "aligned.npz"),
                            slice_sum=al.astype(np.float64).sum((1, 2)),
                            slice_sq=(al.astype(np.float64) ** 2).sum((1, 2)),
                            crop=al[mid, cy - 32:cy + 32, cx - 32:cx + 32].copy())
        if save == 1:
            os.rename(os.path.join(d, "out.xf"), os.path.join(d, "ref.xf"))
        else:
            os.rename(os.path.join(d, "out.txt"), os.path.join(d, "ref.txt"))
        os.remove(out)
    os.remove(mrc)
    with open(os.path.join(d, "case.json"), "w") as fh:
        json.dump({"generator": kw, "thickness": thick, "nproj": nproj, "cmd": cmd[1:],
                   "rc": rc, "wall_s": wall, "perturbation_seed": pert, "save_mode": save},
                  fh, indent=1)
    print(name, "rc", rc, "wall", round(wall, 2), flush=True)
    return rc


# The reference's stdout lines kept as events (printf formats of Transform.cpp:67,92,
# Rotate.cu:328, ProjAlign.cpp:203,485 and Process.cpp:297,305).
_EVENT_PATTERNS = [
    ("img", re.compile(r"^Image\s+(\d+) shift:\s+(\S+),\s+(\S+) px")),
    ("maxerr", re.compile(r"^maxerr:\s+(\S+)")),
    ("axis", re.compile(r"^New tilt axis:\s+(\S+)")),
    ("z0", re.compile(r"^Rot center Z:\s+\S+\s+(\S+)\s+\S+")),
    ("err", re.compile(r"^f(?:Last)?Err\S*:\s+(\S+)")),
    ("meas", re.compile(r"^\s+(-?\d+\.\d\d)\s+(-?\d+\.\d\d)\s+(-?\d+\.\d\d)\s*$")),
]


def parse_log(text):
    events = []
    for line in text.splitlines():
        for kind, pat in _EVENT_PATTERNS:
            m = pat.match(line)
            if not m:
                continue
            vals = [float(v) for v in m.groups()]
            if kind == "img":
                vals[0] = int(vals[0])
            events.append([kind] + vals)
            break
    return events


def parse_txt(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("#"):
                continue
            parts = line.split()
            if len(parts) == 5:
                rows.append([float(v) for v in parts])
    return rows


def write_fixtures(outdir, name):
    d = os.path.join(outdir, name)
    with open(os.path.join(d, "case.json")) as fh:
        case = json.load(fh)
    with open(os.path.join(d, "ref.log"), errors="replace") as fh:
        events = parse_log(fh.read())
    al = np.load(os.path.join(d, "aligned.npz"))
    xf = case.get("save_mode", 0) == 1
    fx = {"case": name, "generator": case["generator"], "thickness": case["thickness"],
          "nproj": case["nproj"], "cmd": case["cmd"],
          "perturbation_seed": case.get("perturbation_seed"), "wall_s": case.get("wall_s"),
          "save_mode": case.get("save_mode", 0),
          "events": events,
          "params": [] if xf else parse_txt(os.path.join(d, "ref.txt")),
          "aligned_slice_sum": al["slice_sum"].tolist(),
          "aligned_slice_sq": al["slice_sq"].tolist()}
    with open(os.path.join(HERE, f"ref_{name}.json"), "w") as fh:
        json.dump(fx, fh)
    ext = "xf" if xf else "txt"
    with open(os.path.join(d, f"ref.{ext}")) as src, \
            open(os.path.join(HERE, f"ref_{name}.{ext}"), "w") as dst:
        dst.write(src.read())
    np.save(os.path.join(HERE, f"ref_{name}_crop.npy"), al["crop"])
    print(name, len(events), "events", flush=True)


def main():
    if sys.argv[1] == "--fixtures":
        outdir = sys.argv[2]
        for n in sys.argv[3:] or list(CASES):
            write_fixtures(outdir, n)
        return 0
    outdir = sys.argv[1]
    names = sys.argv[2:] or list(CASES)
    for n in names:
        case_spec(n)  # unknown names fail before any run
    rc = 0
    for n in names:
        rc |= run_case(outdir, n)
    return rc


if __name__ == "__main__":
    sys.exit(main())
