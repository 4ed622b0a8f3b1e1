"""File-to-file alignment (mf_align_file) against the in-memory entry point (GPU).

mf_align_file streams the MRC stack to the GPU through pinned buffers (8- and
16-bit samples converted there) and streams the aligned stack back to a file.
Its parameters, pass count and output file must be those of mf_align on the same
samples followed by mf_mrc_write, byte for byte.
"""
import os
import sys

import numpy as np
import pytest

from markerfree_b200 import synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_reference_golden import write_mrc  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,descending", [(2, False), (1, True), (0, False)])
def test_align_file_equals_in_memory(ctx, mflib, tmp_path, mode, descending):
    s = synth.make_series(nx=192, ny=160, vol_z=40, n_blobs=70, tilt_min=-42, tilt_max=42,
                          tilt_step=3.0, axis=86.0, shift_sd=3.0, snr=0.8, seed=91,
                          thickness=30)
    stack, angles = s.stack, s.angles
    if mode == 1:
        stack = np.round(stack * 1000.0)
    elif mode == 0:
        lo, hi = stack.min(), stack.max()
        stack = np.round((stack - lo) / (hi - lo) * 255.0)
    if descending:  # the file lists the tilts from +max to -max
        stack, angles = stack[::-1].copy(), angles[::-1].copy()
    src = str(tmp_path / "in.mrc")
    write_mrc(src, stack.astype(np.float32), mode=mode)
    if mode == 0:  # write_mrc knows modes 1 and 2; mode 0 holds unsigned bytes
        with open(src, "r+b") as fh:
            hdr = bytearray(fh.read(1024))
            hdr[12:16] = np.int32(0).tobytes()
            fh.seek(0)
            fh.write(bytes(hdr))
            fh.truncate(1024)
            fh.write(stack.astype(np.uint8).tobytes())
    as_read, m = mflib.mrc_read(src)
    assert m == mode
    kw = dict(offset=1e-4, align_z=30, nproj=10)
    p_mem, out_mem, n_mem = mflib.align(ctx, as_read, angles, want_stack=True, **kw)
    want = str(tmp_path / "mem.mrc")
    mflib.mrc_write(want, out_mem)
    got = str(tmp_path / "file.mrc")
    p_file, n_file = mflib.align_file(ctx, src, angles, got, **kw)
    assert n_file == n_mem
    assert np.array_equal(p_file.shift_x, p_mem.shift_x)
    assert np.array_equal(p_file.shift_y, p_mem.shift_y)
    assert np.array_equal(p_file.rotate, p_mem.rotate)
    with open(got, "rb") as a, open(want, "rb") as b:
        assert a.read() == b.read()
