"""B200 projection-matching alignment (ctypes binding of libmfalign.so).

The library is the product: hand-written sm_100a CUDA kernels plus cuFFT behind
the C ABI declared in include/markerfree.h.  This module loads it from
markerfree_b200/_build/ and mirrors the reference's units of work:

    Series          pre-processed, device-resident tilt series (PreProcess + buf.mrc)
    Series.transform_doit / tilt_axis / find_offset / coarse_align
    Series.projalign_setup / projalign_doit / proj_align / correct_stack
    align()         Process::DoIt minus file I/O
    dev_*()         single kernels on caller-owned device memory

There is no CPU fallback: if the library or a GPU is missing the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libmfalign.so")
CLI_PATH = os.path.join(_HERE, "_build", "Markerfree")

MF_OK = 0
PREC_FP32, PREC_BF16, PREC_FP16 = 0, 1, 2

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_float_p = ctypes.POINTER(ctypes.c_float)


class MfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"markerfree error {code}: {msg}")
        self.code = code


class AlignParamC(ctypes.Structure):
    _fields_ = [("shift_x", _c_float_p), ("shift_y", _c_float_p), ("rotate", _c_float_p),
                ("angle_offset", ctypes.c_float)]


class SeriesDescC(ctypes.Structure):
    _fields_ = [("d_raw", ctypes.c_void_p), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("file_angles", ctypes.c_void_p), ("align_z", ctypes.c_int),
                ("d_out", ctypes.c_void_p)]


class OptionsC(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_float), ("pitch_angle", ctypes.c_float),
                ("zshift", ctypes.c_float), ("thickness", ctypes.c_int),
                ("align_z", ctypes.c_int), ("out_bin", ctypes.c_int), ("gpu", ctypes.c_int),
                ("nproj", ctypes.c_int), ("save_mode", ctypes.c_int),
                ("precision", ctypes.c_int)]


# (name, restype, argtypes) of every entry point in include/markerfree.h
SIGNATURES = [
    ("mf_last_error", ctypes.c_char_p, []),
    ("mf_version", ctypes.c_char_p, []),
    ("mf_context_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_context_destroy", None, [ctypes.c_void_p]),
    ("mf_context_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("mf_context_kernel_launches", ctypes.c_int64, [ctypes.c_void_p]),
    ("mf_series_create", ctypes.c_int, [ctypes.c_void_p, _f32p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _f32p, ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_series_create_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, _f32p,
                                               ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_series_create_preprocessed", ctypes.c_int, [ctypes.c_void_p, _f32p, ctypes.c_int,
                                                     ctypes.c_int, ctypes.c_int, _f32p,
                                                     ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_series_destroy", None, [ctypes.c_void_p]),
    ("mf_series_set_precision", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("mf_series_get_stack", ctypes.c_int, [ctypes.c_void_p, _f32p]),
    ("mf_series_set_angles", ctypes.c_int, [ctypes.c_void_p, _f32p]),
    ("mf_series_get_angles", ctypes.c_int, [ctypes.c_void_p, _f32p]),
    ("mf_series_set_param", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AlignParamC)]),
    ("mf_series_get_param", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AlignParamC)]),
    ("mf_transform_doit", ctypes.c_int, [ctypes.c_void_p, _c_float_p]),
    ("mf_tilt_axis", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_int, _c_float_p]),
    ("mf_find_offset", ctypes.c_int, [ctypes.c_void_p, _c_float_p]),
    ("mf_projalign_setup", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_int,
                                          ctypes.c_int]),
    ("mf_projalign_doit", ctypes.c_int, [ctypes.c_void_p, _c_float_p]),
    ("mf_projalign_z0", ctypes.c_int, [ctypes.c_void_p, _c_float_p]),
    ("mf_projalign_measured", ctypes.c_int, [ctypes.c_void_p, _f32p]),
    ("mf_tilt_axis_scores", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_int,
                                           _c_float_p, _f32p]),
    ("mf_coarse_align", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float]),
    ("mf_proj_align", ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                     _c_int_p]),
    ("mf_correct_stack", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _f32p]),
    ("mf_binned_size", None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p]),
    ("mf_align", ctypes.c_int, [ctypes.c_void_p, _f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                _f32p, ctypes.POINTER(OptionsC), ctypes.POINTER(AlignParamC),
                                ctypes.c_void_p, _c_int_p]),
    ("mf_align_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, _f32p, ctypes.POINTER(OptionsC),
                                       ctypes.POINTER(AlignParamC), ctypes.c_void_p, _c_int_p]),
    ("mf_align_file", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _f32p,
                                     ctypes.POINTER(OptionsC), ctypes.POINTER(AlignParamC),
                                     ctypes.c_char_p, _c_int_p]),
    ("mf_context_set_profiling", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("mf_context_stage_times", ctypes.c_int, [ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_double)]),
    ("mf_context_stage_breakdown", ctypes.c_int, [ctypes.c_void_p,
                                                  ctypes.POINTER(ctypes.c_double)]),
    ("mf_context_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("mf_device_cos_sin", ctypes.c_int, [ctypes.c_void_p, _f32p, ctypes.c_int, _f32p, _f32p]),
    ("mf_context_set_tc_rows", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("mf_context_tc_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.c_int, _c_int_p]),
    ("mf_group_create", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                       ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_group_destroy", None, [ctypes.c_void_p]),
    ("mf_group_doit", ctypes.c_int, [ctypes.c_void_p, _i32p, _f32p]),
    ("mf_group_proj_align", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("mf_group_z0", ctypes.c_int, [ctypes.c_void_p, _f32p]),
    ("mf_align_batch_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                             ctypes.POINTER(SeriesDescC), ctypes.POINTER(OptionsC),
                                             ctypes.POINTER(AlignParamC), ctypes.c_void_p]),
    ("mf_align_many_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p),
                                            ctypes.POINTER(OptionsC),
                                            ctypes.POINTER(AlignParamC),
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    ("mf_server_create", ctypes.c_int, [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    ("mf_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, _f32p,
                                        ctypes.POINTER(OptionsC), ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_int64)]),
    ("mf_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                      ctypes.POINTER(AlignParamC), _c_int_p,
                                      ctypes.POINTER(ctypes.c_double)]),
    ("mf_server_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    ("mf_server_memory", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_int64)]),
    ("mf_debug_fail_device_allocations", None, [ctypes.c_int64, ctypes.c_int64]),
    ("mf_server_destroy", None, [ctypes.c_void_p]),
    ("mf_dev_correct_proj", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    ("mf_find_proj_range", ctypes.c_int, [_f32p, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int,
                                          _i32p]),
    ("mf_dev_reproject", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p]),
    ("mf_dev_reproject_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_void_p]),
    ("mf_dev_measure_shift", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int, ctypes.c_int, _f32p, _c_float_p]),
    ("mf_mrc_info", ctypes.c_int, [ctypes.c_char_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p]),
    ("mf_mrc_read", ctypes.c_int, [ctypes.c_char_p, _f32p]),
    ("mf_mrc_write", ctypes.c_int, [ctypes.c_char_p, _f32p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int]),
    ("mf_read_angles", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, _c_int_p]),
    ("mf_save_param", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(AlignParamC),
                                     _f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_float]),
]

_lib = None


def lib():
    """Load libmfalign.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m markerfree_b200.build` "
                              "(or __graft_entry__.build()) first")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != MF_OK:
        raise MfError(rc, lib().mf_last_error().decode(errors="replace"))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def binned_size(nx: int, ny: int, b: int):
    xb, yb = ctypes.c_int(), ctypes.c_int()
    lib().mf_binned_size(nx, ny, b, ctypes.byref(xb), ctypes.byref(yb))
    return xb.value, yb.value


class Param:
    """AlignParam (Markerfree/src/method/Util.h:14-21) on host arrays."""

    def __init__(self, nz: int):
        self.shift_x = np.zeros(nz, np.float32)
        self.shift_y = np.zeros(nz, np.float32)
        self.rotate = np.zeros(nz, np.float32)
        self.angle_offset = 0.0

    def c(self) -> AlignParamC:
        return AlignParamC(self.shift_x.ctypes.data_as(_c_float_p),
                           self.shift_y.ctypes.data_as(_c_float_p),
                           self.rotate.ctypes.data_as(_c_float_p), float(self.angle_offset))


class Context:
    """One GPU and one stream (the reference's cudaSetDevice, main.cpp:26)."""

    def __init__(self, gpu: int = 0):
        h = ctypes.c_void_p()
        _check(lib().mf_context_create(gpu, ctypes.byref(h)))
        self.h = h

    def sync(self):
        _check(lib().mf_context_sync(self.h))

    def kernel_launches(self) -> int:
        return int(lib().mf_context_kernel_launches(self.h))

    def set_profiling(self, on: bool):
        _check(lib().mf_context_set_profiling(self.h, int(bool(on))))

    def stage_times(self) -> dict:
        """Stage timing accumulated since the previous call (see set_profiling)."""
        out = (ctypes.c_double * 6)()
        _check(lib().mf_context_stage_times(self.h, out))
        keys = ("reproj_ms", "reproj_launches", "xcorr_ms", "passes", "reproj_bytes",
                "reproj_fma")
        return dict(zip(keys, out))

    def device_cos_sin(self, x):
        """CUDA's cosf and sinf of each float32 argument (diagnostic)."""
        x = np.ascontiguousarray(x, np.float32).ravel()
        c = np.zeros_like(x)
        s = np.zeros_like(x)
        _check(lib().mf_device_cos_sin(self.h, x, int(x.size), c, s))
        return c, s

    def stage_breakdown(self) -> dict:
        """Wall ms per alignment stage accumulated since the previous call (stage
        timing on; see set_profiling)."""
        out = (ctypes.c_double * 10)()
        _check(lib().mf_context_stage_breakdown(self.h, out))
        keys = ("prep_ms", "coarse_ms", "axis_ms", "setup_ms", "pass_ms", "output_ms",
                "radon_ms", "radon_launches", "radon_samples", "radon_bytes")
        return dict(zip(keys, out))

    def set_tc_rows(self, rows: int):
        """Image rows per tensor-core tile (64, 128, 256; 0 = automatic)."""
        _check(lib().mf_context_set_tc_rows(self.h, int(rows)))

    def tc_tuning(self) -> list:
        """The autotuner's choices: one dict per (shape, series per launch, precision)."""
        n = ctypes.c_int()
        buf = (ctypes.c_double * (8 * 64))()
        _check(lib().mf_context_tc_tuning(self.h, buf, 64, ctypes.byref(n)))
        rows = []
        for i in range(min(n.value, 64)):
            r = buf[8 * i:8 * i + 8]
            rows.append({"xb": int(r[0]), "yb": int(r[1]), "series": int(r[2]),
                         "precision": int(r[3]), "rows": int(r[4]),
                         "ms_per_launch": {"256": r[5], "128": r[6], "64": r[7]}})
        return rows

    def stream_ptr(self) -> int:
        return int(lib().mf_context_stream(self.h) or 0)

    def close(self):
        # series of this context are released first (the C API requires it)
        for s in list(getattr(self, "_series", ())):
            s.close()
        if getattr(self, "h", None) and _lib is not None:
            _lib.mf_context_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


class Series:
    """A pre-processed tilt series kept in HBM (replaces buf.mrc)."""

    def __init__(self, ctx: Context, raw_stack, file_angles, preprocessed=False):
        """raw_stack in file order (pre-processed on the GPU), or with
        preprocessed=True a stack the reference's PreProcess already treated, in
        ascending angle order (mf_series_create_preprocessed)."""
        import weakref
        raw = _f32(raw_stack)
        self.nz, self.ny, self.nx = raw.shape
        self.ctx = ctx
        self.file_angles = _f32(file_angles)[: self.nz]
        h = ctypes.c_void_p()
        create = lib().mf_series_create_preprocessed if preprocessed else lib().mf_series_create
        _check(create(ctx.h, raw, self.nx, self.ny, self.nz, self.file_angles, ctypes.byref(h)))
        self.h = h
        if not hasattr(ctx, "_series"):
            ctx._series = weakref.WeakSet()
        ctx._series.add(self)

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.mf_series_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    # -- state --
    def stack(self):
        out = np.empty((self.nz, self.ny, self.nx), np.float32)
        _check(lib().mf_series_get_stack(self.h, out))
        return out

    @property
    def angles(self):
        a = np.empty(self.nz, np.float32)
        _check(lib().mf_series_get_angles(self.h, a))
        return a

    @angles.setter
    def angles(self, a):
        _check(lib().mf_series_set_angles(self.h, _f32(a)))

    def get_param(self) -> Param:
        p = Param(self.nz)
        c = p.c()
        _check(lib().mf_series_get_param(self.h, ctypes.byref(c)))
        p.angle_offset = c.angle_offset
        return p

    def set_param(self, p: Param):
        c = p.c()
        _check(lib().mf_series_set_param(self.h, ctypes.byref(c)))

    def set_precision(self, prec: int):
        _check(lib().mf_series_set_precision(self.h, prec))

    # -- stages --
    def transform_doit(self) -> float:
        e = ctypes.c_float()
        _check(lib().mf_transform_doit(self.h, ctypes.byref(e)))
        return e.value

    def tilt_axis(self, rng: float, num: int = 100) -> float:
        a = ctypes.c_float()
        _check(lib().mf_tilt_axis(self.h, rng, num, ctypes.byref(a)))
        return a.value

    def tilt_axis_scores(self, rng: float, num: int = 100):
        """tilt_axis that also returns the score of every candidate."""
        a = ctypes.c_float()
        sc = np.zeros(num, np.float32)
        _check(lib().mf_tilt_axis_scores(self.h, rng, num, ctypes.byref(a), sc))
        return a.value, sc

    def find_offset(self) -> float:
        o = ctypes.c_float()
        _check(lib().mf_find_offset(self.h, ctypes.byref(o)))
        return o.value

    def coarse_align(self, pitch_angle: float = 0.0, offset: float = 0.0):
        _check(lib().mf_coarse_align(self.h, pitch_angle, offset))

    def projalign_setup(self, zshift: float = 0.0, align_z: int = 600, nproj: int = 10):
        _check(lib().mf_projalign_setup(self.h, zshift, align_z, nproj))

    def projalign_doit(self) -> float:
        e = ctypes.c_float()
        _check(lib().mf_projalign_doit(self.h, ctypes.byref(e)))
        return e.value

    @property
    def z0(self) -> float:
        z = ctypes.c_float()
        _check(lib().mf_projalign_z0(self.h, ctypes.byref(z)))
        return z.value

    def projalign_measured(self) -> np.ndarray:
        """(nz, 2) shifts measured in the last pass (un-binned px, before rotation)."""
        xy = np.zeros(2 * self.nz, np.float32)
        _check(lib().mf_projalign_measured(self.h, xy))
        return xy.reshape(-1, 2)

    def proj_align(self, zshift: float = 0.0, align_z: int = 600, nproj: int = 10) -> int:
        n = ctypes.c_int()
        _check(lib().mf_proj_align(self.h, zshift, align_z, nproj, ctypes.byref(n)))
        return n.value

    def correct_stack(self, out_bin: int = 1):
        xo, yo = binned_size(self.nx, self.ny, out_bin)
        out = np.empty((self.nz, yo, xo), np.float32)
        _check(lib().mf_correct_stack(self.h, out_bin, out))
        return out


def align(ctx: Context, raw_stack, file_angles, offset=0.0, pitch_angle=0.0, zshift=0.0,
          align_z=600, out_bin=1, nproj=10, want_stack=True, precision=PREC_FP32):
    """Process::DoIt minus file I/O.  Returns (Param, aligned stack or None, passes)."""
    raw = _f32(raw_stack)
    nz, ny, nx = raw.shape
    p = Param(nz)
    c = p.c()
    o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
    out = None
    ptr = None
    if want_stack:
        xo, yo = binned_size(nx, ny, out_bin)
        out = np.empty((nz, yo, xo), np.float32)
        ptr = out.ctypes.data_as(ctypes.c_void_p)
    n = ctypes.c_int()
    _check(lib().mf_align(ctx.h, raw, nx, ny, nz, _f32(file_angles)[:nz], ctypes.byref(o),
                          ctypes.byref(c), ptr, ctypes.byref(n)))
    p.angle_offset = c.angle_offset
    return p, out, n.value


def align_file(ctx: Context, in_mrc: str, file_angles, out_mrc=None, offset=0.0,
               pitch_angle=0.0, zshift=0.0, align_z=600, out_bin=1, nproj=10,
               precision=PREC_FP32):
    """mf_align_file: MRC stack in, aligned MRC stack out (streamed through pinned
    buffers).  Returns (Param, passes)."""
    nx, ny, nz, _ = mrc_info(in_mrc)
    p = Param(nz)
    c = p.c()
    o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
    n = ctypes.c_int()
    _check(lib().mf_align_file(ctx.h, in_mrc.encode(), _f32(file_angles)[:nz], ctypes.byref(o),
                               ctypes.byref(c), out_mrc.encode() if out_mrc else None,
                               ctypes.byref(n)))
    p.angle_offset = c.angle_offset
    return p, n.value


def align_device(ctx: Context, d_raw, nx, ny, nz, file_angles, d_out, offset=0.0,
                 pitch_angle=0.0, zshift=0.0, align_z=600, out_bin=1, nproj=10,
                 precision=PREC_FP32):
    """mf_align_device: raw stack and aligned output in device memory (torch tensors or
    addresses).  Returns (Param, passes)."""
    p = Param(nz)
    c = p.c()
    o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
    n = ctypes.c_int()
    _check(lib().mf_align_device(ctx.h, _ptr(d_raw), nx, ny, nz, _f32(file_angles)[:nz],
                                 ctypes.byref(o), ctypes.byref(c), _ptr(d_out), ctypes.byref(n)))
    p.angle_offset = c.angle_offset
    return p, n.value


def align_host_ptr(ctx: Context, raw_ptr: int, nx, ny, nz, file_angles, out_ptr: int,
                   offset=0.0, pitch_angle=0.0, zshift=0.0, align_z=600, out_bin=1, nproj=10,
                   precision=PREC_FP32):
    """mf_align on caller-owned host buffers given by address (e.g. pinned memory)."""
    p = Param(nz)
    c = p.c()
    o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
    n = ctypes.c_int()
    f = lib().mf_align
    raw_arr = np.ctypeslib.as_array(ctypes.cast(raw_ptr, _c_float_p), (nz * ny * nx,))
    _check(f(ctx.h, raw_arr, nx, ny, nz, _f32(file_angles)[:nz], ctypes.byref(o),
             ctypes.byref(c), ctypes.c_void_p(out_ptr), ctypes.byref(n)))
    p.angle_offset = c.angle_offset
    return p, n.value


class Group:
    """Projection matching of up to 32 series of one shape in lockstep."""

    def __init__(self, series, zshift=0.0, align_z=600, nproj=10):
        arr = (ctypes.c_void_p * len(series))(*[s.h.value for s in series])
        h = ctypes.c_void_p()
        _check(lib().mf_group_create(arr, len(series), zshift, align_z, nproj, ctypes.byref(h)))
        self.h = h
        self.series = list(series)

    def doit(self, active=None) -> np.ndarray:
        n = len(self.series)
        act = np.ones(n, np.int32) if active is None else np.ascontiguousarray(active, np.int32)
        err = np.zeros(n, np.float32)
        _check(lib().mf_group_doit(self.h, act, err))
        return err

    def proj_align(self) -> np.ndarray:
        passes = np.zeros(len(self.series), np.int32)
        _check(lib().mf_group_proj_align(self.h, passes.ctypes.data_as(ctypes.c_void_p)))
        return passes

    @property
    def z0(self) -> np.ndarray:
        z = np.zeros(len(self.series), np.float32)
        _check(lib().mf_group_z0(self.h, z))
        return z

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.mf_group_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def align_many_device(ctx: Context, d_raws, nx, ny, nz, file_angles, d_outs=None, offset=0.0,
                      pitch_angle=0.0, zshift=0.0, align_z=600, out_bin=1, nproj=10,
                      precision=PREC_FP32):
    """mf_align_many_device: n raw stacks (device tensors or addresses) of one shape.
    Returns (list of Param, passes array)."""
    n = len(d_raws)
    raws = (ctypes.c_void_p * n)(*[_ptr(d).value for d in d_raws])
    angs = [_f32(a)[:nz] for a in file_angles]
    angp = (ctypes.c_void_p * n)(*[a.ctypes.data for a in angs])
    params = [Param(nz) for _ in range(n)]
    cs = (AlignParamC * n)(*[p.c() for p in params])
    outs = None
    if d_outs is not None:
        outs = (ctypes.c_void_p * n)(*[_ptr(d).value for d in d_outs])
    o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
    passes = np.zeros(n, np.int32)
    _check(lib().mf_align_many_device(ctx.h, n, raws, nx, ny, nz, angp, ctypes.byref(o), cs, outs,
                                      passes.ctypes.data_as(ctypes.c_void_p)))
    for p, c in zip(params, cs):
        p.angle_offset = c.angle_offset
    return params, passes


def align_batch_device(ctx: Context, d_raws, file_angles, align_z, d_outs=None, offset=0.0,
                       pitch_angle=0.0, zshift=0.0, out_bin=1, nproj=10, precision=PREC_FP32):
    """mf_align_batch_device: n raw stacks (device tensors, shapes (nz, ny, nx) that
    may differ), per-series angles and slab thicknesses (a sequence, or one value
    for all).  Returns (list of Param, passes array)."""
    n = len(d_raws)
    if not hasattr(align_z, "__len__"):
        align_z = [align_z] * n
    angs = [_f32(a)[:d.shape[0]].copy() for a, d in zip(file_angles, d_raws)]
    descs = (SeriesDescC * n)()
    for i, d in enumerate(d_raws):
        nz, ny, nx = d.shape
        descs[i] = SeriesDescC(_ptr(d).value, nx, ny, nz, angs[i].ctypes.data, int(align_z[i]),
                               _ptr(d_outs[i]).value if d_outs is not None else None)
    params = [Param(d.shape[0]) for d in d_raws]
    cs = (AlignParamC * n)(*[p.c() for p in params])
    # the options' align_z only switches alignment on; each series has its own
    o = OptionsC(offset, pitch_angle, zshift, 0, int(max(align_z)), out_bin, 0, nproj, 0,
                 precision)
    passes = np.zeros(n, np.int32)
    _check(lib().mf_align_batch_device(ctx.h, n, descs, ctypes.byref(o), cs,
                                       passes.ctypes.data_as(ctypes.c_void_p)))
    for p, c in zip(params, cs):
        p.angle_offset = c.angle_offset
    return params, passes


class Server:
    """Continuous-batching request loop (mf_server_*).  Submitted host arrays are
    kept referenced until their job has been waited for."""

    def __init__(self, gpu=0, hbm_budget=0, max_group=8, workers=2, group_wait_ms=50.0):
        h = ctypes.c_void_p()
        _check(lib().mf_server_create(gpu, hbm_budget, max_group, workers, group_wait_ms,
                                      ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, raw, file_angles, out=None, offset=0.0, pitch_angle=0.0, zshift=0.0,
               align_z=600, out_bin=1, nproj=10, precision=PREC_FP32, raw_ptr=None,
               shape=None) -> int:
        """raw: float32 (nz, ny, nx) array, or raw_ptr (host address) with shape."""
        if raw_ptr is None:
            raw = _f32(raw)
            nz, ny, nx = raw.shape
            ptr = raw.ctypes.data
        else:
            nz, ny, nx = shape
            ptr = raw_ptr
        ang = _f32(file_angles)[:nz].copy()
        o = OptionsC(offset, pitch_angle, zshift, 0, align_z, out_bin, 0, nproj, 0, precision)
        jid = ctypes.c_int64()
        outp = None if out is None else ctypes.c_void_p(out.ctypes.data)
        _check(lib().mf_server_submit(self.h, ctypes.c_void_p(ptr), nx, ny, nz, ang,
                                      ctypes.byref(o), outp, ctypes.byref(jid)))
        self._keep[jid.value] = (raw, ang, out, nz)
        return jid.value

    def wait(self, job_id: int, timeout_s: float = 600.0):
        """Returns (Param, passes, latency seconds)."""
        nz = self._keep[job_id][3]
        p = Param(nz)
        c = p.c()
        n = ctypes.c_int()
        lat = ctypes.c_double()
        rc = lib().mf_server_wait(self.h, job_id, timeout_s, ctypes.byref(c), ctypes.byref(n),
                                  ctypes.byref(lat))
        self._keep.pop(job_id, None)
        _check(rc)
        p.angle_offset = c.angle_offset
        return p, n.value, lat.value

    def stats(self) -> dict:
        out = (ctypes.c_double * 8)()
        _check(lib().mf_server_stats(self.h, out))
        keys = ("jobs", "series_per_min", "p50_s", "p99_s", "peak_bytes", "groups",
                "mean_group", "span_s")
        st = dict(zip(keys, out))
        b0, bn, r = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int64()
        _check(lib().mf_server_memory(self.h, ctypes.byref(b0), ctypes.byref(bn),
                                      ctypes.byref(r)))
        st.update(budget_bytes=b0.value, learned_budget_bytes=bn.value, memory_retries=r.value)
        return st

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.mf_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def fail_device_allocations(first, count):
    """Test hook: device allocations number first .. first+count-1, counted from
    this call, fail as if the device were full; count 0 turns it off."""
    lib().mf_debug_fail_device_allocations(int(first), int(count))


def find_proj_range(angles, skip, iproj, nproj):
    a = _f32(angles)
    r = np.zeros(2, np.int32)
    _check(lib().mf_find_proj_range(a, len(a), np.ascontiguousarray(skip, np.uint8), iproj,
                                     nproj, r))
    return int(r[0]), int(r[1])


def _ptr(t):
    """Device pointer of a torch CUDA tensor (or an int address)."""
    if isinstance(t, int):
        return ctypes.c_void_p(t)
    return ctypes.c_void_p(t.data_ptr())


def dev_correct_proj(ctx: Context, d_proj, nx, ny, shift_x, shift_y, tilt_axis, only_shift,
                     binning, random_fill, rweight, d_out):
    _check(lib().mf_dev_correct_proj(ctx.h, _ptr(d_proj), nx, ny, shift_x, shift_y, tilt_axis,
                                     int(only_shift), binning, int(random_fill), int(rweight),
                                     _ptr(d_out)))


def dev_reproject(ctx: Context, d_corr, xb, yb, nz, angles, iproj, istart, iend, thickness,
                  method, d_out):
    _check(lib().mf_dev_reproject(ctx.h, _ptr(d_corr), xb, yb, nz, _f32(angles), iproj, istart,
                                  iend, thickness, method, _ptr(d_out)))


def dev_measure_shift(ctx: Context, d_reproj, d_proj, xb, yb):
    sh = np.zeros(2, np.float32)
    pk = ctypes.c_float()
    _check(lib().mf_dev_measure_shift(ctx.h, _ptr(d_reproj), _ptr(d_proj), xb, yb, sh,
                                      ctypes.byref(pk)))
    return float(sh[0]), float(sh[1]), pk.value


# -- files --
def mrc_info(path: str):
    """(nx, ny, nz, mode) of an MRC file."""
    nx, ny, nz, mode = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().mf_mrc_info(path.encode(), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz),
                             ctypes.byref(mode)))
    return nx.value, ny.value, nz.value, mode.value


def mrc_read(path: str):
    nx, ny, nz, mode = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().mf_mrc_info(path.encode(), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz),
                             ctypes.byref(mode)))
    out = np.empty((nz.value, ny.value, nx.value), np.float32)
    _check(lib().mf_mrc_read(path.encode(), out))
    return out, mode.value


def mrc_write(path: str, data):
    d = _f32(data)
    nz, ny, nx = d.shape
    _check(lib().mf_mrc_write(path.encode(), d, nx, ny, nz))


def read_angles(path: str):
    n = ctypes.c_int()
    _check(lib().mf_read_angles(path.encode(), None, 0, ctypes.byref(n)))
    out = np.empty(n.value, np.float32)
    _check(lib().mf_read_angles(path.encode(), out.ctypes.data_as(ctypes.c_void_p), n.value,
                                ctypes.byref(n)))
    return out


def save_param(output_path: str, mode: int, p: Param, file_angles, raw_nx, raw_ny, out_bin=1,
               elapsed_s=0.0):
    c = p.c()
    a = _f32(file_angles)
    _check(lib().mf_save_param(output_path.encode(), mode, ctypes.byref(c), a, len(a), raw_nx,
                               raw_ny, out_bin, elapsed_s))
