"""The allocation-free re-projection entry point (GPU).

mf_dev_reproject_noalloc serves host programs that cannot let a library allocate
device memory (an acquisition program that has reserved the GPU's memory for its
own buffers, or a real-time loop where cudaMalloc/cudaFree could synchronise the
device).  It keeps its per-neighbour table in a static device array instead of a
scratch buffer.  Called through the C ABI, twice in a row with different
geometry (so the second call must overwrite what the first left in the shared
array), it must give the same output as the allocating entry point
mf_dev_reproject (method 0) and as the oracle's re-projection, and a run of
calls must leave the device's free memory and the memory pool the library
allocates from exactly as they were.

This file is named so that pytest collects it last; it also passes on its own in
a fresh process, where its first call performs the per-device set-up.
"""
import ctypes

import numpy as np
import pytest

from markerfree_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_L2_SUM = 1e-5  # the tolerance of the other re-projection parity tests


def rel_l2(a, b, mask):
    a = np.asarray(a, np.float64)[mask]
    b = np.asarray(b, np.float64)[mask]
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_noalloc_reproject_matches_allocating_entry_point(ctx, mflib):
    import torch
    s = synth.make_series(nx=160, ny=96, vol_z=40, n_blobs=50, tilt_min=-30, tilt_max=30,
                          tilt_step=3.0, axis=86.0, shift_sd=2.0, snr=1.0, seed=31, thickness=30)
    nz, ny, nx = s.stack.shape
    rng = np.random.default_rng(6)
    corr = np.stack([O.correct_proj(s.stack[z], float(rng.normal(0, 2)), float(rng.normal(0, 2)),
                                    86.0, binning=1, rweight=True) for z in range(nz)])
    corr[3, 40, 10:30] = -1e30  # a sentinel run: the invalid masks must agree too
    ang = np.ascontiguousarray(s.angles, np.float32)
    d_corr = torch.from_numpy(corr).cuda()
    torch.cuda.synchronize()
    L = mflib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [(14, 30), (3, 44)]  # (held-out tilt, thickness): different neighbour sets
    for iproj, thick in cases:
        skip = np.ones(nz, np.uint8)
        zt = O.frame_idx_from_tilt(ang)
        lo, hi = sorted((zt, iproj))
        skip[lo:hi + 1] = 0
        skip[iproj] = 1
        i0, i1 = mflib.find_proj_range(ang, skip, iproj, 10)
        assert i0 >= 0
        d_ref = torch.empty((ny, nx), dtype=torch.float32, device="cuda")
        mflib.dev_reproject(ctx, d_corr, nx, ny, nz, ang, iproj, i0, i1, thick, 0, d_ref)
        ctx.sync()
        d_out = torch.full((ny, nx), 3.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc = L.mf_dev_reproject_noalloc(stream, ctypes.c_void_p(d_corr.data_ptr()), nx, ny, nz,
                                        ang, iproj, i0, i1, thick,
                                        ctypes.c_void_p(d_out.data_ptr()))
        assert rc == 0, L.mf_last_error()
        torch.cuda.synchronize()
        want = d_ref.cpu().numpy()
        got = d_out.cpu().numpy()
        valid = want > -1e10
        assert np.array_equal(got > -1e10, valid)
        assert valid.any()
        assert rel_l2(got, want, valid) < REL_L2_SUM
        # and the oracle's re-projection of the same neighbours
        oracle = O.reproject(corr, ang, iproj, i0, i1, thick)
        assert np.array_equal(got > -1e10, oracle > -1e10)
        assert rel_l2(got, oracle, valid) < REL_L2_SUM


def pool_used_bytes(dev=0):
    """Bytes in use in the device's default memory pool (the pool the library's
    allocating entry points draw from), or None without cuda-python."""
    try:
        from cuda.bindings import runtime as rt
    except ImportError:
        return None
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    if err != rt.cudaError_t.cudaSuccess:
        return None
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    return int(used) if err == rt.cudaError_t.cudaSuccess else None


def test_noalloc_reproject_allocates_nothing(ctx, mflib):
    """After a first call (which looks up the table's device address), further calls
    with other geometry change neither the device's free memory nor the bytes in
    use in its default memory pool."""
    import torch
    nz, ny, nx = 21, 64, 96
    rng = np.random.default_rng(8)
    corr = rng.random((nz, ny, nx), dtype=np.float32)
    ang = np.linspace(-30, 30, nz).astype(np.float32)
    d_corr = torch.from_numpy(corr).cuda()
    d_out = torch.empty((ny, nx), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    L = mflib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call(iproj, i0, i1, thick):
        rc = L.mf_dev_reproject_noalloc(stream, ctypes.c_void_p(d_corr.data_ptr()), nx, ny, nz,
                                        ang, iproj, i0, i1, thick,
                                        ctypes.c_void_p(d_out.data_ptr()))
        assert rc == 0, L.mf_last_error()

    call(10, 5, 9, 20)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    used0 = pool_used_bytes()
    for iproj, i0, i1, thick in [(12, 7, 11, 16), (3, 4, 9, 30), (17, 11, 16, 24), (10, 5, 9, 20)]:
        call(iproj, i0, i1, thick)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert pool_used_bytes() == used0


def test_noalloc_reproject_rejects_too_many_neighbours(mflib):
    import torch
    nz = 300
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    L = mflib.lib()
    rc = L.mf_dev_reproject_noalloc(None, ctypes.c_void_p(buf.data_ptr()), 8, 1, nz, ang, 150,
                                    0, 299, 10, ctypes.c_void_p(buf.data_ptr()))
    assert rc == -1
    assert b"maximum of 256" in L.mf_last_error()
