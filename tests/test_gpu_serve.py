"""The serving loop (continuous batching) against each request aligned alone (GPU).

Requests of two shapes arrive while earlier ones are on the GPU; the server
admits them, prepares each on one of its worker streams and projection-matches
prepared requests of one shape together.  Every request's parameters must equal
the ones it gets when aligned alone through mf_align, within the stated
tolerances (0.05 px per-tilt shift, 0.01 degrees tilt axis), and the statistics
must account for every request.
"""
import time

import numpy as np
import pytest

from markerfree_b200 import synth

pytestmark = pytest.mark.gpu

SHIFT_TOL = 0.05
AXIS_TOL = 0.01


def requests():
    out = []
    for i in range(3):
        out.append(synth.make_series(nx=192, ny=160, vol_z=40, n_blobs=70, tilt_min=-42,
                                     tilt_max=42, tilt_step=3.0, axis=85.0 + 2.0 * i,
                                     shift_sd=3.0, snr=0.8, seed=70 + i, thickness=30))
    for i in range(2):
        out.append(synth.make_series(nx=160, ny=128, vol_z=32, n_blobs=50, tilt_min=-30,
                                     tilt_max=30, tilt_step=3.0, axis=88.0 + 2.0 * i,
                                     shift_sd=2.0, snr=1.0, seed=80 + i, thickness=24))
    return out


@pytest.mark.parametrize("prec", [2, 0])
def test_served_results_equal_alone(ctx, mflib, prec):
    reqs = requests()
    kw = [dict(offset=1e-4, align_z=s.thickness, nproj=10, precision=prec) for s in reqs]
    alone = [mflib.align(ctx, s.stack, s.angles, want_stack=True, **k) for s, k in zip(reqs, kw)]
    srv = mflib.Server(gpu=0, hbm_budget=0, max_group=4, workers=2, group_wait_ms=30.0)
    try:
        outs = [np.zeros_like(a[1]) for a in alone]
        ids = []
        for i, (s, k) in enumerate(zip(reqs, kw)):
            ids.append(srv.submit(s.stack, s.angles, out=outs[i], **k))
            time.sleep(0.01 * (i % 2))  # staggered arrivals
        got = [srv.wait(j) for j in ids]
        st = srv.stats()
    finally:
        srv.close()
    assert st["jobs"] == len(reqs)
    assert st["groups"] >= 2  # at most 4 requests per group
    assert st["p99_s"] >= st["p50_s"] > 0
    for i, ((p, passes, lat), (pa, out_a, npa)) in enumerate(zip(got, alone)):
        assert passes == npa, (i, passes, npa)
        assert np.abs(p.rotate - pa.rotate).max() <= AXIS_TOL, i
        assert np.abs(p.shift_x - pa.shift_x).max() <= SHIFT_TOL, i
        assert np.abs(p.shift_y - pa.shift_y).max() <= SHIFT_TOL, i
        if np.array_equal(p.shift_x, pa.shift_x) and np.array_equal(p.shift_y, pa.shift_y):
            assert np.array_equal(outs[i], out_a), i
        assert lat > 0


def test_server_rejects_oversized_request(mflib):
    import ctypes
    srv = mflib.Server(gpu=0, hbm_budget=64 << 20, max_group=2, workers=1)
    try:
        s = synth.make_series(nx=256, ny=256, vol_z=32, n_blobs=20, n_tilts=41, seed=3,
                              thickness=30)
        with pytest.raises(mflib.MfError) as ei:
            srv.submit(s.stack, s.angles, align_z=30)
        assert ei.value.code == -7
    finally:
        srv.close()
    assert ctypes is not None


@pytest.mark.parametrize("first,count", [(5, 3), (40, 2), (120, 4)])
def test_served_requests_survive_a_full_device(ctx, mflib, first, count):
    """Device allocations made to fail (as on a full device) while other requests
    hold memory: the request that met the failure gives its memory back and is
    retried, the learned budget drops, and every result still equals the one the
    request gets alone."""
    reqs = requests()
    kw = [dict(offset=1e-4, align_z=s.thickness, nproj=10, precision=2) for s in reqs]
    alone = [mflib.align(ctx, s.stack, s.angles, want_stack=False, **k)
             for s, k in zip(reqs, kw)]
    srv = mflib.Server(gpu=0, hbm_budget=0, max_group=4, workers=2, group_wait_ms=30.0)
    try:
        # every request is queued before the failures start, so that others hold
        # memory when one meets them (a request alone on a full device fails)
        ids = [srv.submit(s.stack, s.angles, **k) for s, k in zip(reqs, kw)]
        mflib.fail_device_allocations(first, count)
        got = [srv.wait(j) for j in ids]
        st = srv.stats()
    finally:
        mflib.fail_device_allocations(0, 0)
        srv.close()
    assert st["jobs"] == len(reqs)
    assert st["memory_retries"] >= 1
    assert st["learned_budget_bytes"] <= st["budget_bytes"]
    for i, ((p, passes, _), (pa, _, npa)) in enumerate(zip(got, alone)):
        assert passes == npa, (i, passes, npa)
        assert np.abs(p.rotate - pa.rotate).max() <= AXIS_TOL, i
        assert np.abs(p.shift_x - pa.shift_x).max() <= SHIFT_TOL, i
        assert np.abs(p.shift_y - pa.shift_y).max() <= SHIFT_TOL, i


def _pool_bytes_in_use():
    """Bytes of the device's stream-ordered pool (the library's allocations) in use."""
    import torch
    rt = pytest.importorskip("cuda.bindings.runtime")
    torch.cuda.synchronize()
    _, pool = rt.cudaDeviceGetDefaultMemPool(0)
    _, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    return int(used)


@pytest.mark.parametrize("prec", [2, 0])
def test_server_returns_all_device_memory(mflib, prec):
    """Every request's series and every group's buffers go back to the pool: after
    the server closes, the pool holds no more than before it started."""
    reqs = requests()
    before = _pool_bytes_in_use()
    srv = mflib.Server(gpu=0, hbm_budget=0, max_group=4, workers=2, group_wait_ms=20.0)
    try:
        ids = [srv.submit(s.stack, s.angles, offset=1e-4, align_z=s.thickness, nproj=10,
                          precision=prec) for s in reqs]
        for j in ids:
            srv.wait(j)
    finally:
        srv.close()
    assert _pool_bytes_in_use() <= before
