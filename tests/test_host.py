"""Host-side checks that need no GPU: the C ABI loads and exports every
declared entry point, host-only entry points agree with the oracle, the MRC and
angle readers/writers follow the reference's formats, and the command-line tool
validates options like the reference (Markerfree/src/main/opts.h:102-243)."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "markerfree.h")).read()
    return re.findall(r"MF_API\s+[\w\s\*]+?\b(mf_\w+)\s*\(", src)


def test_library_exports_every_declared_symbol(mflib):
    names = declared_symbols()
    assert len(names) >= 30
    L = mflib.lib()
    for n in names:
        assert hasattr(L, n), n
    bound = {s[0] for s in mflib.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound


def test_find_proj_range_matches_oracle(mflib):
    rng = np.random.default_rng(3)
    for nz, step in [(41, 3.0), (61, 2.0), (31, 4.0)]:
        ang = np.linspace(-step * (nz // 2), step * (nz // 2), nz).astype(np.float32)
        for trial in range(20):
            skip = (rng.random(nz) < 0.5).astype(np.uint8)
            ip = int(rng.integers(0, nz))
            for nproj in (1, 3, 10, 20):
                a = mflib.find_proj_range(ang, skip, ip, nproj)
                b = O.find_proj_range(ang, skip, ip, nproj)
                assert a == b


def test_binned_size(mflib):
    for nx, ny, b in [(910, 646, 1), (4096, 4096, 2), (511, 333, 3), (2048, 2048, 4)]:
        assert mflib.binned_size(nx, ny, b) == O.binned_size(nx, ny, b)


def test_mrc_roundtrip_and_header(mflib, tmp_path):
    rng = np.random.default_rng(0)
    d = rng.normal(size=(5, 17, 23)).astype(np.float32)
    d[2, 3, 4] = -1e30  # sentinel: excluded from the middle-slice statistics
    p = str(tmp_path / "x.mrc")
    mflib.mrc_write(p, d)
    back, mode = mflib.mrc_read(p)
    assert mode == 2 and np.array_equal(back, d)
    hdr = np.fromfile(p, np.int32, 256)
    f = hdr.view(np.float32)
    assert list(hdr[:4]) == [23, 17, 5, 2] and list(hdr[7:10]) == [23, 17, 5]
    mid = d[2][d[2] > -1e10]
    assert f[19] == mid.min() and f[20] == mid.max()
    assert abs(f[21] - mid.astype(np.float64).mean()) < 1e-6
    assert os.path.getsize(p) == 1024 + d.nbytes


@pytest.mark.parametrize("mode,dtype", [(0, np.uint8), (1, np.int16), (2, np.float32)])
def test_mrc_read_modes_and_extended_header(mflib, tmp_path, mode, dtype):
    rng = np.random.default_rng(mode)
    d = (rng.random((3, 8, 9)) * 100).astype(dtype)
    nxt = 96
    hdr = np.zeros(256, np.int32)
    hdr[:4] = [9, 8, 3, mode]
    hdr[23] = nxt
    p = str(tmp_path / "m.mrc")
    with open(p, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(b"\x7f" * nxt)
        fh.write(d.tobytes())
    back, m = mflib.mrc_read(p)
    assert m == mode and np.array_equal(back, d.astype(np.float32))


def test_mrc_errors(mflib, tmp_path):
    with pytest.raises(mflib.MfError):
        mflib.mrc_read(str(tmp_path / "missing.mrc"))
    hdr = np.zeros(256, np.int32)
    hdr[:4] = [4, 4, 2, 4]  # complex mode: unsupported, like the reference
    p = str(tmp_path / "c.mrc")
    with open(p, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(b"\0" * 256)
    with pytest.raises(mflib.MfError):
        mflib.mrc_read(p)
    hdr[:4] = [4, 4, 2, 2]
    with open(p, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(b"\0" * 40)  # truncated data
    with pytest.raises(mflib.MfError):
        mflib.mrc_read(p)


def test_read_angles(mflib, tmp_path):
    p = tmp_path / "a.rawtlt"
    p.write_text("-60.0\n -57.5\t-55\n\n12.25 x 3\n")
    a = mflib.read_angles(str(p))
    assert list(a) == [-60.0, -57.5, -55.0, 12.25]  # stops at the first non-number
    with pytest.raises(mflib.MfError):
        mflib.read_angles(str(tmp_path / "none.rawtlt"))


def _cli(mflib, *args):
    r = subprocess.run([mflib.CLI_PATH, *args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout


@pytest.mark.parametrize("args,msg", [
    (["-s", "2"], "Savemode must be 0 or 1."),
    (["-p", "0"], "nProj must be > 0."),
    (["-g", "0,0,0,0,300,1"], ""),
    (["-x"], ""),
])
def test_cli_rejects_bad_options(mflib, args, msg):
    rc, out = _cli(mflib, *args)
    assert rc == 255 and "***WRONG INPUT." in out and msg in out


def test_cli_help(mflib):
    rc, out = _cli(mflib, "-h")
    assert rc == 255 and "[-g O,P,Z,T,A,B,G]" in out and "***WRONG INPUT." in out


def test_cli_missing_input_aborts_cleanly(mflib, tmp_path):
    rc, out = _cli(mflib, "-i", str(tmp_path / "no.mrc"), "-o", str(tmp_path / "o.mrc"), "-a",
                   str(tmp_path / "no.tlt"), "-g", "0,0,0,0,300,1,0")
    assert rc == 0
    assert "[Error] Cannot open input file" in out and "[Abort]" in out
    assert "AlignZ = 300" in out and "nProj = 10" in out


def test_oracle_fft_matches_numpy():
    """The oracle's FP64 FFT (mixed radix + Bluestein) against numpy's pocketfft."""
    import ctypes
    L = O.lib()
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.oc_rfft.argtypes = [dp, dp, ctypes.c_int]
    L.oc_rfft2.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int]
    L.oc_irfft2.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int]
    rng = np.random.default_rng(1)
    for n in (8, 30, 97, 512, 910, 1948, 2046, 2048):
        x = rng.normal(size=n)
        out = np.zeros(2 * (n // 2 + 1))
        L.oc_rfft(x, out, n)
        want = np.fft.rfft(x)
        assert np.abs(out[0::2] + 1j * out[1::2] - want).max() < 1e-9 * n
    for nx, ny in ((64, 48), (910, 8), (30, 1948)):
        x = rng.normal(size=(ny, nx))
        out = np.zeros(2 * (nx // 2 + 1) * ny)
        L.oc_rfft2(np.ascontiguousarray(x), out, nx, ny)
        spec = (out[0::2] + 1j * out[1::2]).reshape(ny, nx // 2 + 1)
        assert np.abs(spec - np.fft.rfft2(x)).max() < 1e-9 * nx * ny
        back = np.zeros((ny, nx))
        L.oc_irfft2(np.ascontiguousarray(out), back, nx, ny)
        assert np.abs(back / (nx * ny) - x).max() < 1e-9


def test_entry_points_reject_bad_arguments_before_touching_the_gpu(mflib):
    """Argument checks of the serving, group, file and tilt-axis entry points come
    before any CUDA call, so they hold on a host without a GPU."""
    import ctypes
    L = mflib.lib()
    srv = ctypes.c_void_p()
    # groups hold 1..32 series, servers run 1..16 workers
    for max_group, workers in ((0, 1), (33, 1), (4, 0), (4, 17)):
        rc = L.mf_server_create(0, 0, max_group, workers, 10.0, ctypes.byref(srv))
        assert rc == -1 and not srv.value, (max_group, workers)
    assert L.mf_server_create(0, 0, 4, 2, 10.0, None) == -1
    assert L.mf_group_create(None, 0, 0.0, 30, 10, ctypes.byref(ctypes.c_void_p())) == -1
    o = mflib.OptionsC(0.0, 0.0, 0.0, 0, 30, 1, 0, 10, 0, 0)
    p = mflib.Param(3)
    a = np.zeros(3, np.float32)
    assert L.mf_align_file(None, b"in.mrc", a, ctypes.byref(o), ctypes.byref(p.c()), None,
                           None) == -1
    assert L.mf_align_file(None, None, a, ctypes.byref(o), ctypes.byref(p.c()), None,
                           None) == -1
    assert L.mf_device_cos_sin(None, a, 3, a, a) == -1
    assert L.mf_projalign_measured(None, a) == -1


def test_oracle_fft_perturbation_probe():
    """oracle.fft_perturb: transform outputs move by at most 2^-24 sqrt(log2 n)
    relative, the same way for the same seed and input, and not at all with seed 0."""
    import ctypes
    L = O.lib()
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.oc_rfft.argtypes = [dp, dp, ctypes.c_int]
    x = np.random.default_rng(2).normal(size=2048)
    outs = []
    try:
        for seed in (0, 7, 7, 8):
            O.fft_perturb(seed)
            o = np.zeros(2 * 1025)
            L.oc_rfft(x, o, 2048)
            outs.append(o)
    finally:
        O.fft_perturb(0)
    rel = np.abs(outs[1] - outs[0]) / np.maximum(np.abs(outs[0]), 1e-300)
    assert 0 < rel.max() <= 2.0 ** -24 * np.sqrt(11) * 1.0001
    assert np.array_equal(outs[1], outs[2]) and not np.array_equal(outs[1], outs[3])
