"""Many series in lockstep (groups) against the same series aligned alone (GPU).

A group runs each stage of a projection-matching pass as one launch over all its
series; each series keeps its own schedule (break rule) through a per-series
active flag.  Each series' result must be the one it gets when aligned alone,
within the stated tolerances (0.05 px per-tilt shift, 0.01 degrees tilt axis),
whatever the other series in the group do.
"""
import numpy as np
import pytest

from markerfree_b200 import synth

pytestmark = pytest.mark.gpu

SHIFT_TOL = 0.05
AXIS_TOL = 0.01


def series_set(n, seed0=40):
    out = []
    for i in range(n):
        # different noise, shifts and axes; same shape
        out.append(synth.make_series(nx=192, ny=160, vol_z=40, n_blobs=70, tilt_min=-42,
                                     tilt_max=42, tilt_step=3.0, axis=84.0 + 3.0 * i,
                                     shift_sd=3.0, snr=0.6 + 0.3 * i, seed=seed0 + i,
                                     thickness=30))
    return out


def to_dev(x):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("prec", [0, 2])
def test_group_matches_alone(ctx, mflib, prec):
    import torch
    ss = series_set(3)
    nz, ny, nx = ss[0].stack.shape
    alone = []
    for s in ss:
        p, _, passes = mflib.align(ctx, s.stack, s.angles, offset=1e-4, align_z=30, nproj=10,
                                   want_stack=False, precision=prec)
        alone.append((p, passes))
    d_raws = [to_dev(s.stack) for s in ss]
    d_outs = [torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda") for _ in ss]
    params, passes = mflib.align_many_device(ctx, d_raws, nx, ny, nz, [s.angles for s in ss],
                                             d_outs, offset=1e-4, align_z=30, nproj=10,
                                             precision=prec)
    for i, (p, (pa, npa)) in enumerate(zip(params, alone)):
        assert passes[i] == npa, (i, passes[i], npa)
        assert np.abs(p.rotate - pa.rotate).max() <= AXIS_TOL
        assert np.abs(p.shift_x - pa.shift_x).max() <= SHIFT_TOL, i
        assert np.abs(p.shift_y - pa.shift_y).max() <= SHIFT_TOL, i
    # the aligned stacks come from the same parameters
    for i, s in enumerate(ss):
        _, out_alone, _ = mflib.align(ctx, s.stack, s.angles, offset=1e-4, align_z=30, nproj=10,
                                      want_stack=True, precision=prec)
        got = d_outs[i].cpu().numpy()
        if np.array_equal(params[i].shift_x, alone[i][0].shift_x) and \
                np.array_equal(params[i].shift_y, alone[i][0].shift_y):
            assert np.array_equal(got, out_alone)


def test_group_pass_with_inactive_series(ctx, mflib):
    """A pass with one series inactive leaves that series untouched and gives the
    other series what a pass of their own gives."""
    ss = series_set(2, seed0=60)
    made = []
    for s in ss:
        ser = mflib.Series(ctx, s.stack, s.angles)
        p = mflib.Param(s.stack.shape[0])
        p.rotate[:] = 86.0
        ser.set_param(p)
        made.append(ser)
    g = mflib.Group(made, 0.0, 30, 10)
    e1 = g.doit([1, 1])
    before = made[1].get_param()
    e2 = g.doit([1, 0])
    after = made[1].get_param()
    assert np.array_equal(before.shift_x, after.shift_x)
    assert np.array_equal(before.shift_y, after.shift_y)
    g.close()
    # series 0 alone through the single-series path for the same two passes
    s0 = ss[0]
    ser = mflib.Series(ctx, s0.stack, s0.angles)
    p = mflib.Param(s0.stack.shape[0])
    p.rotate[:] = 86.0
    ser.set_param(p)
    ser.projalign_setup(0.0, 30, 10)
    a1 = ser.projalign_doit()
    a2 = ser.projalign_doit()
    assert abs(a1 - e1[0]) < 1e-3 and abs(a2 - e2[0]) < 1e-3
    q0 = made[0].get_param()
    qa = ser.get_param()
    assert np.abs(q0.shift_x - qa.shift_x).max() < 1e-3
    assert np.abs(q0.shift_y - qa.shift_y).max() < 1e-3


def uneven_set():
    """Three series that differ in image size, tilt count, tilt range and slab
    thickness (the uneven batches of many-series alignment)."""
    return [
        (synth.make_series(nx=192, ny=160, vol_z=40, n_blobs=70, tilt_min=-42, tilt_max=42,
                           tilt_step=3.0, axis=85.0, shift_sd=3.0, snr=0.8, seed=71,
                           thickness=30), 30),
        (synth.make_series(nx=160, ny=128, vol_z=32, n_blobs=50, tilt_min=-30, tilt_max=30,
                           tilt_step=3.0, axis=88.0, shift_sd=2.5, snr=1.0, seed=72,
                           thickness=24), 24),
        (synth.make_series(nx=256, ny=224, vol_z=48, n_blobs=90, tilt_min=-48, tilt_max=48,
                           tilt_step=4.0, axis=83.0, shift_sd=3.0, snr=0.7, seed=73,
                           thickness=40), 40),
    ]


@pytest.mark.parametrize("prec", [0, 2])
def test_uneven_group_matches_alone(ctx, mflib, prec):
    """Series of different sizes, tilt counts and thicknesses aligned in one group
    (one launch per stage over all of them) give what each gets alone."""
    import torch
    ss = uneven_set()
    alone = []
    for s, az in ss:
        p, out, passes = mflib.align(ctx, s.stack, s.angles, offset=1e-4, align_z=az, nproj=10,
                                     want_stack=True, precision=prec)
        alone.append((p, out, passes))
    d_raws = [to_dev(s.stack) for s, _ in ss]
    d_outs = [torch.empty(s.stack.shape, dtype=torch.float32, device="cuda") for s, _ in ss]
    params, passes = mflib.align_batch_device(ctx, d_raws, [s.angles for s, _ in ss],
                                              [az for _, az in ss], d_outs, offset=1e-4,
                                              nproj=10, precision=prec)
    for i, (p, (pa, out_alone, npa)) in enumerate(zip(params, alone)):
        assert passes[i] == npa, (i, passes[i], npa)
        assert np.abs(p.rotate - pa.rotate).max() <= AXIS_TOL
        assert np.abs(p.shift_x - pa.shift_x).max() <= SHIFT_TOL, i
        assert np.abs(p.shift_y - pa.shift_y).max() <= SHIFT_TOL, i
        if np.array_equal(p.shift_x, pa.shift_x) and np.array_equal(p.shift_y, pa.shift_y):
            assert np.array_equal(d_outs[i].cpu().numpy(), out_alone)
