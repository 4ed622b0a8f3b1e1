"""The alignment on the GPU against the reference program's own output.

tests/golden/ holds what the unmodified reference (built from its sources, run
on a B200) printed and wrote for seeded synthetic series
(tests/golden/make_reference_golden.py; every case passes -g 1e-4,0,0,0,T,1,0
-p NPROJ, so the offset search is skipped).

Stage by stage, the GPU path must reproduce the reference's printed values
until the first data-dependent decision that a rounding difference can flip:
the largest shift of each coarse stretch-correlation pass, the tilt axes of the
coarse searches, and the largest shift and rotation centre of the first
projection-matching pass.

The reference is itself sensitive: the same input multiplied by
1 + 1e-6 * U(-1, 1) (cases "<name>_p1" ... "<name>_p6", seeds 1-6) already moves
the shifts it prints for the first projection-matching passes by 0.01 px, and
its final tilt axis by up to 2.5 degrees and its shifts by up to 0.9 px on the
low-SNR series (near-tied axis candidates flip, and nearest-neighbour
re-correction amplifies the change in later passes); on the high-SNR hi384
series five of its seven runs end on the same axis and the other two 0.017
degrees away.  So each printed stage value is compared with the closest of the
reference's runs, and the final parameters must agree with one of its runs
within max(0.01 deg, its axis spread) and max(0.05 px, its shift spread): the
stated tolerances wherever the reference itself is stable.
"""
import itertools
import json
import os

import numpy as np
import pytest

from markerfree_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
AXIS_TOL = 0.01   # degrees
SHIFT_TOL = 0.05  # px
PRINT_TOL = 0.0051 + 0.005  # values printed with 2 decimals, plus float noise


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


def reference_logs(name):
    """The reference's outputs for the case and for each of its perturbations."""
    out = []
    for suffix in [""] + [f"_p{k}" for k in range(1, 10)]:
        p = os.path.join(GOLD, f"ref_{name}{suffix}.json")
        if os.path.exists(p):
            with open(p) as f:
                out.append(json.load(f))
    return out


def reference_runs(name):
    return [np.array(g["params"], np.float64) for g in reference_logs(name)]


def events(g, kind):
    return [e[1:] for e in g["events"] if e[0] == kind]


def closest(value, logs, kind, i):
    """|value - printed| for the reference run that printed the closest value."""
    return min(abs(value - events(g, kind)[i][0]) for g in logs)


@pytest.mark.parametrize("name", ["c1s256", "c1s256b", "cfg1", "hi384", "bin2", "cfg2"])
def test_stages_match_reference_log(ctx, mflib, name):
    g, s, angles = load(name)
    logs = reference_logs(name)
    ser = mflib.Series(ctx, s.stack, angles)
    same = True  # our trajectory still equals the reference's (to its printed digits)
    for i in range(3):
        e = ser.transform_doit()
        if i == 0 or (same and len(logs) > 1):
            assert closest(e, logs, "maxerr", i) < PRINT_TOL, (i, e, events(g, "maxerr")[i])
        elif same and closest(e, logs, "maxerr", i) >= PRINT_TOL:
            # One reference run only (the 2048^2 series, SNR 0.05): there the second
            # stretch pass lands on a neighbouring integer peak for a few high-tilt
            # pairs (a near-tie; the FP64 oracle takes the same peaks as this
            # library), so the comparison ends at that first near-tied decision.
            same = False
        ax = ser.tilt_axis(180.0 / (i + 1))
        if i == 0:
            assert closest(ax, logs, "axis", 0) < PRINT_TOL, (ax, events(g, "axis")[0])
        same = same and closest(ax, logs, "axis", i) < PRINT_TOL
    if not same:
        return  # a near-tied axis candidate flipped; the final-parameter test covers the rest
    # -g 1e-4: no offset search, the offset is applied to the angles
    ser.angles = angles + np.float32(1e-4)
    p = ser.get_param()
    p.shift_x[:] = 0
    p.shift_y[:] = 0
    ser.set_param(p)
    ser.projalign_setup(0.0, g["thickness"], g["nproj"])
    e = ser.projalign_doit()
    assert closest(e, logs, "err", 0) < PRINT_TOL, (e, [events(r, "err")[0] for r in logs])
    ser.projalign_doit()
    assert closest(ser.z0, logs, "z0", 1) < 0.02


@pytest.mark.parametrize("name", ["c1s256", "c1s256b", "cfg1", "hi384", "bin2"])
def test_final_parameters_within_reference_spread(ctx, mflib, name):
    g, s, angles = load(name)
    runs = reference_runs(name)
    assert len(runs) >= 4, "perturbed reference runs missing"
    ax_spread = max(abs(a[0, 1] - b[0, 1]) for a, b in itertools.combinations(runs, 2))
    sh_spread = max(np.abs(a[:, 2:4] - b[:, 2:4]).max() for a, b in itertools.combinations(runs, 2))
    ax_tol = max(AXIS_TOL, ax_spread)
    sh_tol = max(SHIFT_TOL, sh_spread)
    p, _, passes = mflib.align(ctx, s.stack, angles, offset=1e-4, pitch_angle=0.0, zshift=0.0,
                               align_z=g["thickness"], out_bin=1, nproj=g["nproj"],
                               want_stack=False)
    best = None
    for r in runs:
        d_ax = float(np.abs(p.rotate.astype(np.float64) - r[:, 1]).max())
        d_sh = float(max(np.abs(p.shift_x - r[:, 2]).max(), np.abs(p.shift_y - r[:, 3]).max()))
        score = max(d_ax / ax_tol, d_sh / sh_tol)
        if best is None or score < best[0]:
            best = (score, d_ax, d_sh)
    print(f"{name}: passes {passes}, axis {p.rotate[0]:.4f}; reference axes "
          f"{[round(r[0, 1], 4) for r in runs]}, spread {ax_spread:.4f} deg / {sh_spread:.4f} px; "
          f"closest run: d_axis {best[1]:.4f} deg, d_shift {best[2]:.4f} px")
    assert best[0] <= 1.0, best


def printed_pass(g, nz, k):
    """(nz - 1, 3) rows (tilt angle, x shift, y shift) the run printed in projection-
    matching pass k."""
    return np.array(events(g, "meas")[k * (nz - 1):(k + 1) * (nz - 1)])


@pytest.mark.parametrize("name", ["hi384", "c1s256", "cfg1", "bin2", "cfg2"])
def test_first_passes_match_reference_prints(ctx, mflib, name):
    """Every per-tilt shift the reference printed in its first two projection-
    matching passes, against one of its runs: within print rounding plus the
    spread of the runs that follow that run's trajectory."""
    g, s, angles = load(name)
    logs = reference_logs(name)
    nz = len(angles)
    ser = mflib.Series(ctx, s.stack, angles)
    for i in range(3):
        ser.transform_doit()
        ax = ser.tilt_axis(180.0 / (i + 1))
        if closest(ax, logs, "axis", i) >= PRINT_TOL:
            pytest.skip("coarse axis candidate flipped: later stages follow another trajectory")
    ang = angles + np.float32(1e-4)
    ser.angles = ang
    p = ser.get_param()
    p.shift_x[:] = 0
    p.shift_y[:] = 0
    ser.set_param(p)
    ser.projalign_setup(0.0, g["thickness"], g["nproj"])
    near = list(range(len(logs)))  # runs on the trajectory being followed
    for k in range(2):
        ser.projalign_doit()
        m = ser.projalign_measured()
        dev = {}
        for i in near:
            pr = printed_pass(logs[i], nz, k)
            z = [int(np.argmin(np.abs(ang - a))) for a in pr[:, 0]]
            dev[i] = float(np.abs(m[z] - pr[:, 1:]).max())
        best = min(dev, key=dev.get)
        ref = printed_pass(logs[best], nz, k)[:, 1:]
        near = [i for i in near if np.abs(printed_pass(logs[i], nz, k)[:, 1:] - ref).max() < 0.1]
        spread = max(float(np.abs(printed_pass(logs[i], nz, k)[:, 1:] -
                                  printed_pass(logs[j], nz, k)[:, 1:]).max())
                     for i in near for j in near)
        print(f"{name} pass {k + 1}: deviation {dev[best]:.4f} from run {best}, "
              f"spread of the {len(near)} runs on its trajectory {spread:.3f}")
        assert dev[best] < PRINT_TOL + spread, (k, dev, spread)


def aligned_runs():
    out = []
    for name in ["c1s256", "c1s256b", "cfg1", "hi384", "bin2", "cfg2"]:
        for g in reference_logs(name):
            k = g.get("perturbation_seed")
            out.append(name if k is None else f"{name}_p{k}")
    return out


@pytest.mark.parametrize("run", aligned_runs())
def test_aligned_stack_matches_reference_output(ctx, mflib, run):
    """The library's output writer (mf_correct_stack: resampling, random fill), given
    the parameters the reference wrote to its .txt, against the reference's own
    aligned stack (Process.cpp:329-372): the 64 x 64 crop of the middle slice is
    equal bit for bit on every pixel whose source pixel the printed parameters
    determine, relative L2 over the whole crop within 1e-5, and every slice sum
    within the rounding that the undetermined pixels allow."""
    import sys as _sys
    _sys.path.insert(0, GOLD)
    from make_reference_golden import perturbed
    from test_oracle_golden import determined_pixels
    with open(os.path.join(GOLD, f"ref_{run}.json")) as f:
        g = json.load(f)
    s = case_series(g)
    angles = np.array([float(f"{a:.2f}") for a in s.angles], np.float32)
    seed = g.get("perturbation_seed")
    raw = s.stack if seed is None else perturbed(s.stack, seed)
    nz, ny, nx = raw.shape
    params = np.array(g["params"], np.float64)
    ser = mflib.Series(ctx, raw, angles)
    p = mflib.Param(nz)
    p.rotate[:] = params[:, 1]
    p.shift_x[:] = params[:, 2]
    p.shift_y[:] = params[:, 3]
    ser.set_param(p)
    al = ser.correct_stack(1)
    ser.close()
    crop_ref = np.load(os.path.join(GOLD, f"ref_{run}_crop.npy"))
    mid, cy, cx = nz // 2, ny // 2, nx // 2
    crop = al[mid, cy - 32:cy + 32, cx - 32:cx + 32]
    det = determined_pixels(params, nx, ny, mid, cy - 32, cx - 32, 64, 64)
    assert det.mean() > 0.95
    assert np.array_equal(crop[det], crop_ref[det])
    rel = np.linalg.norm((crop - crop_ref).astype(np.float64)) / np.linalg.norm(crop_ref)
    assert rel <= 1e-5, rel
    sums = al.astype(np.float64).sum((1, 2))
    ref_sums = np.array(g["aligned_slice_sum"])
    assert float(np.abs(sums - ref_sums).max() / np.abs(ref_sums).max()) < 2e-4


def test_cli_matches_reference_parameter_file(mflib, tmp_path):
    """The drop-in program, run with the reference's command line on the input the
    reference was given (hi384, -g 0.0001,0,0,0,80,1,0 -p 10 -s 0; Process.cpp:34-92,
    SaveParam.cpp:185-262): its .txt has the reference's layout line for line, and
    every row's axis and shifts agree with one of the reference's runs within
    max(0.01 deg, their axis spread) and max(0.05 px, their shift spread)."""
    import subprocess
    import sys as _sys
    _sys.path.insert(0, GOLD)
    from make_reference_golden import parse_txt, write_mrc
    g, s, angles = load("hi384")
    runs = reference_runs("hi384")
    mrc = str(tmp_path / "in.mrc")
    tlt = str(tmp_path / "in.rawtlt")
    out = str(tmp_path / "out.mrc")
    write_mrc(mrc, s.stack)
    with open(tlt, "w") as fh:
        for a in s.angles:
            fh.write(f"{a:.2f}\n")
    cli = os.path.join(os.path.dirname(HERE), "markerfree_b200", "_build", "Markerfree")
    r = subprocess.run([cli, "-i", mrc, "-o", out, "-a", tlt, "-g",
                        f"0.0001,0,0,0,{g['thickness']},1,0", "-p", str(g["nproj"]), "-s", "0"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    mine = open(str(tmp_path / "out.txt")).read().splitlines()
    ref = open(os.path.join(GOLD, "ref_hi384.txt")).read().splitlines()
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        if a.startswith("Elapsed time"):
            assert b.startswith("Elapsed time")
        elif a.startswith("#") or ":" in a:
            assert a == b
    rows = np.array(parse_txt(str(tmp_path / "out.txt")), np.float64)
    assert np.array_equal(rows[:, 0], runs[0][:, 0]) and np.allclose(rows[:, 4], runs[0][:, 4])
    ax_spread = max(abs(a[0, 1] - b[0, 1]) for a, b in itertools.combinations(runs, 2))
    sh_spread = max(np.abs(a[:, 2:4] - b[:, 2:4]).max() for a, b in itertools.combinations(runs, 2))
    score = min(max(np.abs(rows[:, 1] - r[:, 1]).max() / max(AXIS_TOL, ax_spread),
                    np.abs(rows[:, 2:4] - r[:, 2:4]).max() / max(SHIFT_TOL, sh_spread))
                for r in runs)
    assert score <= 1.0, score
    # the aligned stack it wrote: float32 MRC of the input's size
    nx, ny, nz, mode = mflib.mrc_info(out)
    assert (nx, ny, nz, mode) == (s.stack.shape[2], s.stack.shape[1], s.stack.shape[0], 2)
