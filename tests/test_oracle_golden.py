"""The CPU oracle against the reference program's own outputs (CPU only).

The reference was run on seeded synthetic series (tests/golden/make_reference_golden.py)
and its log and parameter file were kept as fixtures.  The oracle is pinned where
the reference's trajectory is still deterministic: every per-image shift of the
first coarse (stretch cross-correlation) pass, the first tilt-axis searches, and
every per-tilt shift of the first projection-matching pass.  Later passes of the
reference re-correct images with nearest-neighbour rounding of accumulated
shifts, so float-level differences between cuFFT and any other FFT can flip a
pixel and the trajectories drift apart by a few hundredths of a pixel; those are
compared with a tolerance.
"""
import json
import os

import numpy as np
import pytest

from markerfree_b200 import synth
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
# the reference log prints shifts with 2 decimals
PRINT_TOL = 0.0051 + 0.005


def case_series(g):
    """The series a fixture's run was generated from (make_reference_golden's cases)."""
    if "config" in g["generator"]:
        return synth.config(g["generator"]["config"])
    return synth.make_series(thickness=g["thickness"], nproj=g["nproj"], **g["generator"])


def load(name):
    with open(os.path.join(GOLD, f"ref_{name}.json")) as f:
        g = json.load(f)
    s = case_series(g)
    angles = np.array([float(f"{a:.2f}") for a in s.angles], np.float32)
    return g, s, angles


def events(g, kind):
    return [e for e in g["events"] if e[0] == kind]


def reference_logs(name):
    """The reference's outputs for the case and for each of its perturbations
    (input x (1 + 1e-6 U(-1, 1)), seeds 1-6): equally valid reference results."""
    out = []
    for suffix in [""] + [f"_p{k}" for k in range(1, 10)]:
        p = os.path.join(GOLD, f"ref_{name}{suffix}.json")
        if os.path.exists(p):
            with open(p) as f:
                out.append(json.load(f))
    return out


def pass_deviation(meas, ang, ref):
    """Largest |measured - printed| over one pass's printed per-tilt shifts."""
    return max(max(abs(meas[int(np.argmin(np.abs(ang - e[1]))), 0] - e[2]),
                   abs(meas[int(np.argmin(np.abs(ang - e[1]))), 1] - e[3])) for e in ref)


def printed_pass(g, nz, k):
    """(nz - 1, 2) shifts the run printed in projection-matching pass k."""
    return np.array([e[2:] for e in events(g, "meas")[k * (nz - 1):(k + 1) * (nz - 1)]])


def pass_tolerance(logs, best, nz, k):
    """Print rounding plus the spread of pass k among the reference runs that follow
    run `best`'s trajectory (printed shifts within 0.1 px of it): how far apart
    the reference's own results for the same series lie."""
    ref = printed_pass(logs[best], nz, k)
    near = [printed_pass(g, nz, k) for g in logs]
    near = [m for m in near if np.abs(m - ref).max() < 0.1]
    spread = max(float(np.abs(a - b).max()) for a in near for b in near)
    return PRINT_TOL + spread


def transform_passes(g):
    passes, cur = [], {}
    for e in g["events"]:
        if e[0] == "img":
            cur[e[1] - 1] = (e[2], e[3])
        elif e[0] == "maxerr":
            passes.append(cur)
            cur = {}
    return passes


@pytest.mark.parametrize("name", ["c1s256", "c1s256b", "bin2"])
def test_first_coarse_pass_matches_reference(name):
    g, s, angles = load(name)
    st = O.preprocess(s.stack, angles)
    p = O.Param(len(angles))
    t = O.Transform(st, angles, p)
    e = t.doit()
    mx, my = t.measured()
    ref = transform_passes(g)[0]
    assert len(ref) == len(angles) - 1
    for z, (rx, ry) in ref.items():
        assert abs(mx[z] - rx) < PRINT_TOL and abs(my[z] - ry) < PRINT_TOL, (z, mx[z], my[z], rx, ry)
    assert abs(e - events(g, "maxerr")[0][1]) < PRINT_TOL
    # the first tilt-axis search (range 180) sees identical shifts
    ax = O.tilt_axis(st, angles, p, 180.0)
    assert abs(ax - events(g, "axis")[0][1]) < 0.0051


def test_coarse_stage_and_first_projection_pass_match_reference():
    g, s, angles = load("c1s256")
    nz = len(angles)
    st = O.preprocess(s.stack, angles)
    p = O.Param(nz)
    t = O.Transform(st, angles, p)
    axes = []
    for i in (1, 2, 3):
        t.doit()
        axes.append(O.tilt_axis(st, angles, p, 180.0 / i))
    ref_axes = [e[1] for e in events(g, "axis")[:3]]
    assert np.allclose(axes, ref_axes, atol=0.0051), (axes, ref_axes)
    # -g 1e-4,...: the offset search is skipped and the offset applied
    ang = angles + np.float32(0.0001)
    p.shift_x[:] = 0
    p.shift_y[:] = 0
    pa = O.ProjAlign(st, ang, p, 0.0, g["thickness"], g["nproj"])
    logs = reference_logs("c1s256")
    assert len(logs) >= 7
    err = pa.doit()
    meas = pa.measured()
    # the first pass agrees, tilt by tilt, with one of the reference's runs
    dev = [pass_deviation(meas, ang, events(r, "meas")[: nz - 1]) for r in logs]
    best = int(np.argmin(dev))
    assert dev[best] < pass_tolerance(logs, best, nz, 0), dev
    # the runs on that trajectory (first-pass prints within 0.1 px of run `best`)
    near = [g for g in logs
            if np.abs(printed_pass(g, nz, 0) - printed_pass(logs[best], nz, 0)).max() < 0.1]
    assert min(abs(err - events(g, "err")[0][1]) for g in near) < PRINT_TOL
    # second pass: rotation centre z and largest shift as those runs printed them
    err2 = pa.doit()
    assert min(abs(pa.z0 - events(g, "z0")[1][1]) for g in near) < PRINT_TOL
    tol2 = pass_tolerance(logs, best, nz, 1)
    assert min(abs(err2 - events(g, "err")[1][1]) for g in near) < tol2
    meas2 = pa.measured()
    worst = min(pass_deviation(meas2, ang, events(g, "meas")[nz - 1: 2 * (nz - 1)]) for g in near)
    assert worst < tol2, (worst, tol2)


def test_parameter_file_format_matches_reference_example(mflib, tmp_path):
    """mf_save_param reproduces the reference's .txt layout byte for byte."""
    src = os.path.join(GOLD, "ts1_align_reference.txt")
    lines = open(src).read().splitlines()
    rows = [l.split() for l in lines[3:44]]
    nz = len(rows)
    p = mflib.Param(nz)
    p.rotate[:] = [float(r[1]) for r in rows]
    p.shift_x[:] = [float(r[2]) for r in rows]
    p.shift_y[:] = [float(r[3]) for r in rows]
    p.angle_offset = 5.0
    angles = np.array([float(r[4]) for r in rows], np.float32)
    out = str(tmp_path / "TS_1_align.mrc")
    mflib.save_param(out, 0, p, angles, 910, 646, 1, 45.851048)
    mine = open(str(tmp_path / "TS_1_align.txt")).read().splitlines()
    assert mine == lines


def test_xf_writer_layout(mflib, tmp_path):
    nz = 5
    p = mflib.Param(nz)
    p.rotate[:] = 94.68
    p.shift_x[:] = np.arange(nz)
    p.shift_y[:] = -np.arange(nz)
    angles = np.linspace(40, -40, nz).astype(np.float32)  # descending: rows reversed
    mflib.save_param(str(tmp_path / "a.mrc"), 1, p, angles, 910, 646)
    txt = open(str(tmp_path / "a.xf")).read().splitlines()
    assert len(txt) == nz
    th = np.float32(94.68) * np.pi / np.float32(180.0)
    c, s = np.float32(np.cos(th)), np.float32(np.sin(th))
    first = [float(v) for v in txt[0].split()]
    assert abs(first[0] - c) < 1e-3 and abs(first[1] - s) < 1e-3
    # inv: the first row is the last internal tilt (shift x = 4)
    cx = cy = np.float32(910 / 2.0)
    T1 = -4.0 - cx + c * cx - s * cy
    T2 = 4.0 - cy + s * cx + c * cy
    assert abs(first[4] - (T1 * c + T2 * s - cx + c * cx + s * cy)) < 2e-3
    assert txt[0].endswith(" ")  # the reference's trailing blank before the newline


def test_fp64_reprojection_agrees_with_fp32_restatement():
    """The FP64 re-projection (the reference for the precision error statements)
    takes the same index decisions as the FP32 restatement and differs from it by
    FP32 rounding only."""
    s = synth.make_series(nx=120, ny=96, vol_z=24, n_blobs=40, tilt_min=-24, tilt_max=24,
                          tilt_step=4.0, axis=86.0, shift_sd=2.0, snr=1.0, seed=9, thickness=20)
    rng = np.random.default_rng(1)
    corr = np.stack([O.correct_proj(s.stack[z], float(rng.normal(0, 2)), float(rng.normal(0, 2)),
                                    86.0, binning=1, rweight=True)
                     for z in range(s.stack.shape[0])])
    w32 = O.reproject(corr, s.angles, 9, 3, 8, 20)
    w64 = O.reproject_f64(corr, s.angles, 9, 3, 8, 20)
    valid = w64 > -1e10
    assert valid.any()
    assert np.array_equal(valid, w32 > -1e10)
    err = np.linalg.norm(w32[valid] - w64[valid]) / np.linalg.norm(w64[valid])
    assert err < 1e-6, err


def test_first_passes_on_the_stable_series_match_reference():
    """hi384 (SNR 4), on which the reference's own runs agree: the oracle follows its
    coarse stage to the printed digits and every per-tilt shift of its first two
    projection-matching passes to print rounding plus the runs' own spread."""
    g, s, angles = load("hi384")
    logs = reference_logs("hi384")
    nz = len(angles)
    st = O.preprocess(s.stack, angles)
    p = O.Param(nz)
    t = O.Transform(st, angles, p)
    for i in (1, 2, 3):
        e = t.doit()
        ax = O.tilt_axis(st, angles, p, 180.0 / i)
        assert min(abs(e - events(r, "maxerr")[i - 1][1]) for r in logs) < PRINT_TOL
        assert min(abs(ax - events(r, "axis")[i - 1][1]) for r in logs) < PRINT_TOL
    ang = angles + np.float32(0.0001)
    p.shift_x[:] = 0
    p.shift_y[:] = 0
    pa = O.ProjAlign(st, ang, p, 0.0, g["thickness"], g["nproj"])
    for k in range(2):
        pa.doit()
        meas = pa.measured()
        dev = [pass_deviation(meas, ang, events(r, "meas")[k * (nz - 1):(k + 1) * (nz - 1)])
               for r in logs]
        best = int(np.argmin(dev))
        assert dev[best] < pass_tolerance(logs, best, nz, k), (k, dev)


# ---------------------------------------------------------------------------
# Aligned output stack (Process::CorrectStack, Markerfree/src/main/Process.cpp:329-372;
# CorrStack.cu:142-179): the reference kept a 64 x 64 crop of the middle slice of
# its aligned stack and the per-slice sums of the whole stack.
SHIFT_PRINT = 0.0005   # the .txt prints shifts with 3 decimals
ROT_PRINT = 0.00005    # and the tilt axis with 4


def run_input(g):
    """The stack the reference was given for run g (perturbed for "_p<k>" runs)."""
    import sys as _sys
    _sys.path.insert(0, GOLD)
    from make_reference_golden import perturbed
    s = case_series(g)
    angles = np.array([float(f"{a:.2f}") for a in s.angles], np.float32)
    seed = g.get("perturbation_seed")
    return (s.stack if seed is None else perturbed(s.stack, seed)), angles


def determined_pixels(params, nx, ny, z, y0, x0, h, w, margin=SHIFT_PRINT + 2e-4):
    """Pixels of the crop whose nearest source pixel the printed parameters fix:
    the source coordinate x + 0.5 stays on one side of an integer over the
    print-rounding interval of the shifts and the axis (CorrStack.cu:160-170)."""
    th = np.deg2rad(params[z, 1])
    r = np.hypot(w, h)
    m = margin + r * np.deg2rad(ROT_PRINT)
    yy, xx = np.mgrid[y0:y0 + h, x0:x0 + w].astype(np.float64)
    u, v = xx + 0.5 - nx * 0.5, yy + 0.5 - ny * 0.5
    X = u * np.cos(th) - v * np.sin(th) + params[z, 2] + nx * 0.5 + 0.5
    Y = u * np.sin(th) + v * np.cos(th) + params[z, 3] + ny * 0.5 + 0.5
    return (np.abs(X - np.round(X)) > m) & (np.abs(Y - np.round(Y)) > m)


def reference_aligned_runs():
    out = []
    for name in ["c1s256", "c1s256b", "cfg1", "hi384", "bin2"]:
        for g in reference_logs(name):
            sfx = "" if g.get("perturbation_seed") is None else f"_p{g['perturbation_seed']}"
            out.append(f"{name}{sfx}")
    return out


@pytest.mark.parametrize("run", reference_aligned_runs())
def test_aligned_stack_matches_reference_output(run):
    """The oracle's output writer, given the parameters the reference wrote, against
    the reference's own aligned stack: the crop is equal bit for bit on every pixel
    whose source pixel the printed parameters determine (all but a few per cent),
    and every slice sum agrees to the rounding those undetermined pixels allow."""
    with open(os.path.join(GOLD, f"ref_{run}.json")) as f:
        g = json.load(f)
    raw, angles = run_input(g)
    nz, ny, nx = raw.shape
    st = O.preprocess(raw, angles)
    params = np.array(g["params"], np.float64)
    p = O.Param(nz)
    p.rotate[:] = params[:, 1]
    p.shift_x[:] = params[:, 2]
    p.shift_y[:] = params[:, 3]
    al = O.correct_stack(st, p, 1)
    crop_ref = np.load(os.path.join(GOLD, f"ref_{run}_crop.npy"))
    mid, cy, cx = nz // 2, ny // 2, nx // 2
    crop = al[mid, cy - 32:cy + 32, cx - 32:cx + 32]
    det = determined_pixels(params, nx, ny, mid, cy - 32, cx - 32, 64, 64)
    assert det.mean() > 0.95, det.mean()
    assert np.array_equal(crop[det], crop_ref[det])
    rel = np.linalg.norm((crop - crop_ref).astype(np.float64)) / np.linalg.norm(crop_ref)
    assert rel <= 1e-5, rel
    sums = al.astype(np.float64).sum((1, 2))
    ref_sums = np.array(g["aligned_slice_sum"])
    srel = float(np.abs(sums - ref_sums).max() / np.abs(ref_sums).max())
    print(f"{run}: {det.mean():.4f} of the crop determined; crop rel-L2 {rel:.2e}, "
          f"largest slice-sum difference {srel:.2e}")
    assert srel < 2e-4


def test_xf_matches_reference_output(mflib, tmp_path):
    """The .xf writer (SaveParam::SaveXf, SaveParam.cpp:15-53, with its height = X
    quirk and -s 1's reversed row order) given the parameters the reference wrote
    for hi384, against the .xf the reference wrote for the same input with -s 1:
    same rows in the same order and layout, values within the rounding of the
    .txt's printed parameters (shifts 3 decimals, axis 4)."""
    import re
    g, s, angles = load("hi384")
    params = np.array(g["params"], np.float64)
    nz = len(angles)
    p = mflib.Param(nz)
    p.rotate[:] = params[:, 1]
    p.shift_x[:] = params[:, 2]
    p.shift_y[:] = params[:, 3]
    out = str(tmp_path / "hi384.mrc")
    mflib.save_param(out, 1, p, angles, s.stack.shape[2], s.stack.shape[1])
    mine = open(str(tmp_path / "hi384.xf")).read().splitlines()
    ref = open(os.path.join(GOLD, "ref_hi384_s1.xf")).read().splitlines()
    assert len(mine) == len(ref) == nz
    pat = re.compile(r"^( *-?\d+\.\d{3} {2}){5} *-?\d+\.\d{3} $")
    for a, b in zip(mine, ref):
        assert pat.match(a) and pat.match(b), (a, b)
        va = np.array([float(v) for v in a.split()])
        vb = np.array([float(v) for v in b.split()])
        assert np.abs(va - vb).max() <= 0.0021, (a, b)


def test_bin2_first_projection_pass_matches_reference():
    """The 3072 px series that the reference matches at bin 2 (ProjAlign.cpp:57-61,
    slab 100 / 2 = 50): the oracle follows its coarse stage and every per-tilt
    shift of its first projection-matching pass, to print rounding plus the spread
    of the reference's runs on that trajectory."""
    g, s, angles = load("bin2")
    logs = reference_logs("bin2")
    nz = len(angles)
    st = O.preprocess(s.stack, angles)
    p = O.Param(nz)
    t = O.Transform(st, angles, p)
    for i in (1, 2, 3):
        e = t.doit()
        ax = O.tilt_axis(st, angles, p, 180.0 / i)
        assert min(abs(e - events(r, "maxerr")[i - 1][1]) for r in logs) < PRINT_TOL
        assert min(abs(ax - events(r, "axis")[i - 1][1]) for r in logs) < PRINT_TOL
    ang = angles + np.float32(0.0001)
    p.shift_x[:] = 0
    p.shift_y[:] = 0
    pa = O.ProjAlign(st, ang, p, 0.0, g["thickness"], g["nproj"])
    pa.doit()
    meas = pa.measured()
    dev = [pass_deviation(meas, ang, events(r, "meas")[: nz - 1]) for r in logs]
    best = int(np.argmin(dev))
    assert dev[best] < pass_tolerance(logs, best, nz, 0), dev
