"""Mixed-precision (FP16/BF16 operand, FP32 accumulate) tensor-core re-projection
against the CPU oracle (GPU).

The tensor-core path applies the same banded operator as the FP32 path to a
16-bit copy of the corrected stack, so its error against the FP32 oracle is the
16-bit rounding of the operands.  Index work still has to agree exactly: which
columns are invalid (-1e30) and which 128-row tiles fall back to the exact FP32
gather because a neighbour row holds a sentinel or an FP16-overflowing value.
"""
import numpy as np
import pytest

from markerfree_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# relative L2 error of a re-projected image against the FP32 oracle
REL_L2_TC = {2: 2e-3, 3: 1.5e-2}   # method 2 = FP16 operands, 3 = BF16 operands
REL_L2_EXACT = 1e-5                # tiles recomputed by the exact FP32 gather
SHIFT_TOL_MIXED = 0.05             # px, per-tilt shifts of a mixed-precision pass


def rel_l2(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def to_dev(x):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    torch.cuda.synchronize()
    return t


@pytest.fixture(scope="module")
def tall():
    """A 200 x 384 series: two 128-column x-tiles (the second partial) and three
    128-row tiles."""
    s = synth.make_series(nx=200, ny=384, vol_z=40, n_blobs=90, tilt_min=-28, tilt_max=28,
                          tilt_step=4.0, axis=86.0, shift_sd=3.0, snr=1.0, seed=21,
                          thickness=30)
    rng = np.random.default_rng(4)
    corr = np.stack([O.correct_proj(s.stack[z], float(rng.normal(0, 2)),
                                    float(rng.normal(0, 2)), 86.0, binning=1, rweight=True)
                     for z in range(s.stack.shape[0])])
    return s, corr


def neighbours(ang, iproj, nproj=10):
    nz = len(ang)
    skip = np.ones(nz, np.uint8)
    zt = O.frame_idx_from_tilt(ang)
    lo, hi = sorted((zt, iproj))
    skip[lo:hi + 1] = 0
    skip[iproj] = 1
    return O.find_proj_range(ang, skip, iproj, nproj)


@pytest.mark.parametrize("rows", [64, 128, 256])
@pytest.mark.parametrize("method", [2, 3])
@pytest.mark.parametrize("iproj,thick", [(10, 30), (2, 40), (13, 12)])
def test_tc_reproject_matches_oracle(ctx, mflib, tall, method, rows, iproj, thick):
    import torch
    s, corr = tall
    nz, yb, xb = corr.shape
    ang = s.angles
    i0, i1 = neighbours(ang, iproj)
    assert i0 >= 0
    want = O.reproject(corr, ang, iproj, i0, i1, thick)
    d_out = torch.full((yb, xb), 7.0, dtype=torch.float32, device="cuda")
    ctx.set_tc_rows(rows)
    try:
        mflib.dev_reproject(ctx, to_dev(corr), xb, yb, nz, ang, iproj, i0, i1, thick, method,
                            d_out)
    finally:
        ctx.set_tc_rows(0)
    got = d_out.cpu().numpy()
    assert np.isfinite(got).all()
    valid = want > -1e10
    assert np.array_equal(got > -1e10, valid)
    assert valid.any()
    assert rel_l2(got, want, valid) < REL_L2_TC[method]


@pytest.mark.parametrize("method", [2, 3])
def test_tc_sentinel_tiles_use_exact_path(ctx, mflib, tall, method):
    import torch
    s, corr = tall
    nz, yb, xb = corr.shape
    ang = s.angles
    iproj = 10
    i0, i1 = neighbours(ang, iproj)
    c = corr.copy()
    c[i0 + 1, 150, 40:60] = -1e30  # invalid pixels in a neighbour row of row tile 1
    want = O.reproject(c, ang, iproj, i0, i1, 30)
    d_out = torch.empty((yb, xb), dtype=torch.float32, device="cuda")
    mflib.dev_reproject(ctx, to_dev(c), xb, yb, nz, ang, iproj, i0, i1, 30, method, d_out)
    got = d_out.cpu().numpy()
    valid = want > -1e10
    assert np.array_equal(got > -1e10, valid)
    tile1 = np.zeros_like(valid)
    tile1[128:256] = True
    assert rel_l2(got, want, valid & tile1) < REL_L2_EXACT
    assert rel_l2(got, want, valid & ~tile1) < REL_L2_TC[method]


def test_tc_fp16_overflow_uses_exact_path(ctx, mflib, tall):
    import torch
    s, corr = tall
    nz, yb, xb = corr.shape
    ang = s.angles
    iproj = 10
    i0, i1 = neighbours(ang, iproj)
    c = corr.copy()
    c[i1, 300, 100] = 2.0e5  # beyond the FP16 range: row tile 2 goes exact
    want = O.reproject(c, ang, iproj, i0, i1, 30)
    d_out = torch.empty((yb, xb), dtype=torch.float32, device="cuda")
    mflib.dev_reproject(ctx, to_dev(c), xb, yb, nz, ang, iproj, i0, i1, 30, 2, d_out)
    got = d_out.cpu().numpy()
    assert np.isfinite(got).all()
    valid = want > -1e10
    assert rel_l2(got[256:], want[256:], valid[256:]) < REL_L2_EXACT
    assert rel_l2(got, want, valid) < REL_L2_TC[2]


@pytest.mark.parametrize("prec", [1, 2])
def test_mixed_precision_pass_matches_oracle(ctx, mflib, prec):
    """Two projection-matching passes with 16-bit operands against the FP32 oracle:
    every per-tilt shift within 0.05 px."""
    s0 = synth.make_series(nx=160, ny=128, vol_z=40, n_blobs=60, tilt_min=-28, tilt_max=28,
                           tilt_step=4.0, axis=86.0, shift_sd=3.0, snr=1.0, seed=5,
                           thickness=30)
    nz = s0.stack.shape[0]
    st = O.preprocess(s0.stack, s0.angles)
    s = mflib.Series(ctx, s0.stack, s0.angles)
    s.set_precision(prec)
    p = mflib.Param(nz)
    p.rotate[:] = 86.0
    s.set_param(p)
    po = O.Param(nz)
    po.rotate[:] = 86.0
    pa = O.ProjAlign(st, s0.angles, po, 0.0, 30, 10)
    s.projalign_setup(0.0, 30, 10)
    for k in range(2):
        e_o = pa.doit()
        e_g = s.projalign_doit()
        g = s.get_param()
        assert abs(e_g - e_o) < SHIFT_TOL_MIXED, (k, e_g, e_o)
        assert np.abs(g.shift_x - po.shift_x).max() < SHIFT_TOL_MIXED
        assert np.abs(g.shift_y - po.shift_y).max() < SHIFT_TOL_MIXED


# relative L2 error of each path's re-projection against the FP64 restatement
# (same discrete geometry, every value accumulated in FP64)
REL_L2_VS_FP64 = {0: 1e-6, 1: 1e-6, 2: 2e-3, 3: 1.5e-2}


@pytest.mark.parametrize("iproj,thick", [(10, 30), (2, 40)])
def test_precision_errors_against_fp64(ctx, mflib, tall, iproj, thick):
    """The error of every re-projection path against the FP64 oracle: the exact
    FP32 gather (0), the FP32 banded operator (1), FP16 (2) and BF16 (3) operands
    with FP32 accumulation.  The valid-pixel masks are identical."""
    import torch
    s, corr = tall
    nz, yb, xb = corr.shape
    ang = s.angles
    i0, i1 = neighbours(ang, iproj)
    want = O.reproject_f64(corr, ang, iproj, i0, i1, thick)
    valid = want > -1e10
    assert valid.any()
    d_corr = to_dev(corr)
    errs = {}
    for method in (0, 1, 2, 3):
        d_out = torch.full((yb, xb), 7.0, dtype=torch.float32, device="cuda")
        mflib.dev_reproject(ctx, d_corr, xb, yb, nz, ang, iproj, i0, i1, thick, method, d_out)
        got = d_out.cpu().numpy()
        assert np.array_equal(got > -1e10, valid), method
        errs[method] = rel_l2(got, want, valid)
    print("relative L2 against FP64:", {k: f"{v:.2e}" for k, v in errs.items()})
    for method, e in errs.items():
        assert e < REL_L2_VS_FP64[method], (method, e)


@pytest.mark.parametrize("prec", [0, 2, 1])
def test_pass_shift_errors_against_fp64_oracle(ctx, mflib, prec):
    """The per-tilt shift error, in px, of two projection-matching passes in each
    precision (mf_precision 0 = FP32, 2 = FP16, 1 = BF16 operands) against the oracle whose
    re-projection accumulates in FP64: within 0.05 px, and stated."""
    s0 = synth.make_series(nx=160, ny=128, vol_z=40, n_blobs=60, tilt_min=-28, tilt_max=28,
                           tilt_step=4.0, axis=86.0, shift_sd=3.0, snr=1.0, seed=5,
                           thickness=30)
    nz = s0.stack.shape[0]
    st = O.preprocess(s0.stack, s0.angles)
    s = mflib.Series(ctx, s0.stack, s0.angles)
    s.set_precision(prec)
    p = mflib.Param(nz)
    p.rotate[:] = 86.0
    s.set_param(p)
    po = O.Param(nz)
    po.rotate[:] = 86.0
    pa = O.ProjAlign(st, s0.angles, po, 0.0, 30, 10)
    pa.set_f64(True)
    s.projalign_setup(0.0, 30, 10)
    worst = 0.0
    for _ in range(2):
        pa.doit()
        s.projalign_doit()
        g = s.get_param()
        worst = max(worst, float(np.abs(g.shift_x - po.shift_x).max()),
                    float(np.abs(g.shift_y - po.shift_y).max()))
    print(f"precision {prec}: largest per-tilt shift error against FP64 {worst:.4f} px")
    assert worst < SHIFT_TOL_MIXED, worst


@pytest.mark.parametrize("prec", [0, 2, 1])
def test_tilt_axis_error_against_fp64_oracle(ctx, mflib, prec):
    """The tilt axis, in degrees, that each precision (mf_precision 0 = FP32, 2 = FP16,
    1 = BF16 operands) finds after two projection-matching passes (the 20-degree
    refinement of Process::mProjAlign, Process.cpp:283-296), against the oracle
    whose re-projection accumulates in FP64 and whose search sees the FP64 path's
    shifts: within 0.01 degrees, and stated."""
    s0 = synth.make_series(nx=192, ny=192, vol_z=48, n_blobs=90, tilt_min=-45, tilt_max=45,
                           tilt_step=3.0, axis=87.0, shift_sd=3.0, snr=4.0, seed=21,
                           thickness=40)
    nz = s0.stack.shape[0]
    st = O.preprocess(s0.stack, s0.angles)
    s = mflib.Series(ctx, s0.stack, s0.angles)
    s.set_precision(prec)
    p = mflib.Param(nz)
    p.rotate[:] = 86.0
    s.set_param(p)
    po = O.Param(nz)
    po.rotate[:] = 86.0
    pa = O.ProjAlign(st, s0.angles, po, 0.0, 40, 10)
    pa.set_f64(True)
    s.projalign_setup(0.0, 40, 10)
    for _ in range(2):
        pa.doit()
        s.projalign_doit()
    ax_o, sc_o = O.tilt_axis_scores(st, s0.angles, po, 20.0)
    ax_g = s.tilt_axis(20.0)
    top = np.sort(sc_o)[-2:]
    err = abs(ax_g - ax_o)
    print(f"precision {prec}: tilt axis {ax_g:.4f} against FP64 {ax_o:.4f}: error {err:.4f} deg "
          f"(oracle's best two candidate scores {top[1]:.6f}, {top[0]:.6f})")
    assert err <= 0.01, err
