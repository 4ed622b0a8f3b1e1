"""ctypes binding of the CPU oracle (oracle/oc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by bench.py's
CPU-baseline leg as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_SOURCES = [os.path.join(_HERE, "oc_oracle.cpp"), os.path.join(_HERE, "oc_fft.cpp")]

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OcParam(ctypes.Structure):
    _fields_ = [("shift_x", ctypes.POINTER(ctypes.c_float)),
                ("shift_y", ctypes.POINTER(ctypes.c_float)),
                ("rotate", ctypes.POINTER(ctypes.c_float)),
                ("angle_offset", ctypes.c_float)]


def build(force: bool = False) -> str:
    """Compile the oracle shared library (g++, OpenMP) if it is missing or stale."""
    newest = max(os.path.getmtime(s) for s in _SOURCES + [os.path.join(_HERE, "oc_fft.hpp"),
                                                           os.path.join(_HERE, "oc_oracle.hpp")])
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < newest:
        os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
        # no contraction except the explicit std::fmaf calls, which -mfma makes single
        # instructions
        cmd = ["g++", "-O2", "-mfma", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
               "-std=c++17",
               "-o", _LIB_PATH] + _SOURCES
        subprocess.check_call(cmd)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oc_frame_idx_from_tilt.argtypes = [ctypes.c_int, _f32p, ctypes.c_float]
        L.oc_projalign_set_f64.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oc_projalign_set_f64.restype = None
        L.oc_trig_set.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p]
        L.oc_trig_set.restype = None
        L.oc_fft_perturb.argtypes = [ctypes.c_ulonglong]
        L.oc_fft_perturb.restype = None
        L.oc_trig_record.argtypes = [ctypes.c_int]
        L.oc_trig_record.restype = None
        L.oc_trig_recorded.argtypes = [_f32p, ctypes.c_int]
        L.oc_find_ref_index.argtypes = [ctypes.c_int, _f32p, ctypes.c_int]
        L.oc_preprocess.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p]
        L.oc_binned_size.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int)] * 2
        L.oc_correct_proj.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, _f32p]
        L.oc_find_proj_range.argtypes = [_f32p, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int,
                                         _i32p]
        L.oc_reproject.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p]
        L.oc_reproject_f64.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")]
        L.oc_measure_shift.argtypes = [_f32p, _f32p, ctypes.c_int, ctypes.c_int, _f32p,
                                       ctypes.POINTER(ctypes.c_float)]
        L.oc_projalign_create.restype = ctypes.c_void_p
        L.oc_projalign_create.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                          ctypes.POINTER(OcParam), ctypes.c_float, ctypes.c_int,
                                          ctypes.c_int]
        L.oc_projalign_doit.restype = ctypes.c_float
        L.oc_projalign_doit.argtypes = [ctypes.c_void_p]
        L.oc_projalign_z0.restype = ctypes.c_float
        L.oc_projalign_z0.argtypes = [ctypes.c_void_p]
        L.oc_projalign_bin.argtypes = [ctypes.c_void_p]
        L.oc_projalign_measured.argtypes = [ctypes.c_void_p, _f32p]
        L.oc_projalign_destroy.argtypes = [ctypes.c_void_p]
        L.oc_tilt_axis.restype = ctypes.c_float
        L.oc_tilt_axis.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                   ctypes.POINTER(OcParam), ctypes.c_float, ctypes.c_int]
        L.oc_tilt_axis_scores.restype = ctypes.c_float
        L.oc_tilt_axis_scores.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                          ctypes.POINTER(OcParam), ctypes.c_float, ctypes.c_int,
                                          _f32p]
        L.oc_transform_create.restype = ctypes.c_void_p
        L.oc_transform_create.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                          ctypes.POINTER(OcParam)]
        L.oc_transform_doit.restype = ctypes.c_float
        L.oc_transform_doit.argtypes = [ctypes.c_void_p]
        L.oc_transform_destroy.argtypes = [ctypes.c_void_p]
        L.oc_transform_measured.argtypes = [ctypes.c_void_p, _f32p, _f32p]
        L.oc_find_offset.restype = ctypes.c_float
        L.oc_find_offset.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                                     ctypes.POINTER(OcParam)]
        L.oc_correct_stack.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(OcParam), ctypes.c_int, _f32p]
        L.oc_align.restype = ctypes.c_int
        L.oc_align.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p,
                               ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                               ctypes.c_int, ctypes.c_int, ctypes.POINTER(OcParam),
                               ctypes.c_void_p, ctypes.c_int]
        _lib = L
    return _lib


class Param:
    """Host AlignParam mirror (Markerfree/src/method/Util.h:14-21)."""

    def __init__(self, nz: int):
        self.shift_x = np.zeros(nz, np.float32)
        self.shift_y = np.zeros(nz, np.float32)
        self.rotate = np.zeros(nz, np.float32)
        self.c = OcParam()
        fp = ctypes.POINTER(ctypes.c_float)
        self.c.shift_x = self.shift_x.ctypes.data_as(fp)
        self.c.shift_y = self.shift_y.ctypes.data_as(fp)
        self.c.rotate = self.rotate.ctypes.data_as(fp)
        self.c.angle_offset = 0.0

    def copy(self) -> "Param":
        q = Param(self.shift_x.size)
        q.shift_x[:] = self.shift_x
        q.shift_y[:] = self.shift_y
        q.rotate[:] = self.rotate
        q.angle_offset = self.angle_offset
        return q

    @property
    def angle_offset(self) -> float:
        return float(self.c.angle_offset)

    @angle_offset.setter
    def angle_offset(self, v: float):
        self.c.angle_offset = float(v)

    def ref(self):
        return ctypes.byref(self.c)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def fft_perturb(seed: int):
    """Perturb every FFT output of the oracle by a relative 2^-24 sqrt(log2 n) at most
    (deterministic per seed; 0 turns it off): a probe of how far single-precision
    transform rounding, such as cuFFT's, can move the results."""
    lib().oc_fft_perturb(ctypes.c_ulonglong(int(seed)))


def trig_set(x, c, s):
    """Use these cos/sin values (CUDA's, measured on the GPU) for these float
    arguments instead of the correctly rounded ones; trig_set([], [], []) clears."""
    x, c, s = _f32(x), _f32(c), _f32(s)
    lib().oc_trig_set(int(x.size), x, c, s)


def trig_clear():
    e = np.zeros(0, np.float32)
    lib().oc_trig_set(0, e, e, e)


class trig_recording:
    """Context manager collecting the float arguments cos/sin are evaluated at;
    .args holds them afterwards."""

    def __enter__(self):
        lib().oc_trig_record(1)
        self.args = None
        return self

    def __exit__(self, *exc):
        lib().oc_trig_record(0)
        n = lib().oc_trig_recorded(np.zeros(1, np.float32), 0)
        out = np.zeros(max(n, 1), np.float32)
        lib().oc_trig_recorded(out, n)
        self.args = out[:n]
        return False


def frame_idx_from_tilt(angles, tilt=0.0):
    a = _f32(angles)
    return lib().oc_frame_idx_from_tilt(len(a), a, tilt)


def binned_size(nx, ny, b):
    xb, yb = ctypes.c_int(), ctypes.c_int()
    lib().oc_binned_size(nx, ny, b, ctypes.byref(xb), ctypes.byref(yb))
    return xb.value, yb.value


def preprocess(raw, angles):
    raw = _f32(raw)
    nz, ny, nx = raw.shape
    out = np.empty_like(raw)
    lib().oc_preprocess(raw, nx, ny, nz, _f32(angles), out)
    return out


def correct_proj(proj, shift_x, shift_y, tilt_axis, only_shift=False, binning=1,
                 random_fill=True, rweight=True):
    proj = _f32(proj)
    ny, nx = proj.shape
    xb, yb = binned_size(nx, ny, binning)
    out = np.empty((yb, xb), np.float32)
    lib().oc_correct_proj(proj, nx, ny, shift_x, shift_y, tilt_axis, int(only_shift), binning,
                          int(random_fill), int(rweight), out)
    return out


def find_proj_range(angles, skip, iproj, nproj):
    a = _f32(angles)
    sk = np.ascontiguousarray(skip, dtype=np.uint8)
    r = np.zeros(2, np.int32)
    lib().oc_find_proj_range(a, len(a), sk, iproj, nproj, r)
    return int(r[0]), int(r[1])


def reproject(corr, angles, iproj, istart, iend, thickness):
    corr = _f32(corr)
    nz, yb, xb = corr.shape
    out = np.empty((yb, xb), np.float32)
    lib().oc_reproject(corr, xb, yb, nz, _f32(angles), iproj, istart, iend, thickness, out)
    return out


def reproject_f64(corr, angles, iproj, istart, iend, thickness):
    """reproject() with every value accumulated in FP64 and the same FP32 index
    decisions: the reference for the error statements of each precision."""
    corr = _f32(corr)
    nz, yb, xb = corr.shape
    out = np.empty((yb, xb), np.float64)
    lib().oc_reproject_f64(corr, xb, yb, nz, _f32(angles), iproj, istart, iend, thickness, out)
    return out


def measure_shift(reproj, proj):
    r, p = _f32(reproj), _f32(proj)
    yb, xb = r.shape
    sh = np.zeros(2, np.float32)
    pk = ctypes.c_float()
    lib().oc_measure_shift(r, p, xb, yb, sh, ctypes.byref(pk))
    return float(sh[0]), float(sh[1]), float(pk.value)


def tilt_axis(stack, angles, param: Param, rng: float, num: int = 100):
    stack = _f32(stack)
    nz, ny, nx = stack.shape
    return lib().oc_tilt_axis(stack, nx, ny, nz, _f32(angles), param.ref(), rng, num)


def tilt_axis_scores(stack, angles, param: Param, rng: float, num: int = 100):
    stack = _f32(stack)
    nz, ny, nx = stack.shape
    sc = np.zeros(num, np.float32)
    ax = lib().oc_tilt_axis_scores(stack, nx, ny, nz, _f32(angles), param.ref(), rng, num, sc)
    return ax, sc


def find_offset(stack, angles, param: Param):
    stack = _f32(stack)
    nz, ny, nx = stack.shape
    return lib().oc_find_offset(stack, nx, ny, nz, _f32(angles), param.ref())


def correct_stack(stack, param: Param, out_bin=1):
    stack = _f32(stack)
    nz, ny, nx = stack.shape
    xo, yo = binned_size(nx, ny, out_bin)
    out = np.empty((nz, yo, xo), np.float32)
    lib().oc_correct_stack(stack, nx, ny, nz, param.ref(), out_bin, out)
    return out


class ProjAlign:
    """Mirror of ProjAlign (Markerfree/src/method/ProjAlign.h:11-78)."""

    def __init__(self, stack, angles, param: Param, zshift=0.0, align_z=600, nproj=10):
        self._stack = _f32(stack)
        self._angles = _f32(angles)
        nz, ny, nx = self._stack.shape
        self.param = param
        self._h = lib().oc_projalign_create(self._stack, nx, ny, nz, self._angles, param.ref(),
                                            zshift, align_z, nproj)

    def doit(self) -> float:
        return lib().oc_projalign_doit(self._h)

    def set_f64(self, on: bool = True):
        """Re-project in FP64 in later passes (the reference for precision errors)."""
        lib().oc_projalign_set_f64(self._h, int(bool(on)))

    @property
    def z0(self) -> float:
        return lib().oc_projalign_z0(self._h)

    def measured(self):
        """(nz, 2) shifts measured in the last pass, un-binned px, before rotation."""
        xy = np.zeros(2 * self._stack.shape[0], np.float32)
        lib().oc_projalign_measured(self._h, xy)
        return xy.reshape(-1, 2)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oc_projalign_destroy(self._h)
            self._h = None


class Transform:
    """Mirror of Transform (Markerfree/src/method/Transform.h:10-31)."""

    def __init__(self, stack, angles, param: Param):
        self._stack = _f32(stack)
        self._angles = _f32(angles)
        nz, ny, nx = self._stack.shape
        self._h = lib().oc_transform_create(self._stack, nx, ny, nz, self._angles, param.ref())

    def doit(self) -> float:
        return lib().oc_transform_doit(self._h)

    def measured(self):
        """Per-image shifts of the last pass (the reference's "Image %d shift" lines)."""
        n = self._stack.shape[0]
        x, y = np.zeros(n, np.float32), np.zeros(n, np.float32)
        lib().oc_transform_measured(self._h, x, y)
        return x, y

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oc_transform_destroy(self._h)
            self._h = None


def align(raw, file_angles, offset=0.0, pitch_angle=0.0, zshift=0.0, align_z=600, out_bin=1,
          nproj=10, want_stack=True, verbose=False):
    """Whole pipeline (Process::DoIt minus file I/O).  Returns (param, aligned, passes)."""
    raw = _f32(raw)
    nz, ny, nx = raw.shape
    p = Param(nz)
    out = None
    ptr = None
    if want_stack:
        xo, yo = binned_size(nx, ny, out_bin)
        out = np.empty((nz, yo, xo), np.float32)
        ptr = out.ctypes.data_as(ctypes.c_void_p)
    passes = lib().oc_align(raw, nx, ny, nz, _f32(file_angles), offset, pitch_angle, zshift,
                            align_z, out_bin, nproj, p.ref(), ptr, int(verbose))
    return p, out, passes
