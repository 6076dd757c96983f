"""ctypes bindings for the checkers (test infrastructure only).

* ``Oracle`` wraps ``oracle/_build/liboracle.so`` - the C restatement of the
  reference's per-frame path (``oracle/wema_oracle.c``).
* ``Reference`` wraps ``oracle/_ref/libref_harness.so`` - the reference's own
  library sources compiled by ``oracle/Makefile`` and driven through the
  reference's public C API (``oracle/ref_harness.c``).  It exists only where
  the reference was compiled (it is built in the development container and
  travels with the repository snapshot); ``Reference.available()`` says so.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libref_harness.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class _Cfg(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fps", C.c_float),
                ("amp", C.c_float), ("f_low", C.c_float), ("f_high", C.c_float),
                ("window", C.c_int), ("edge_aware", C.c_int), ("bilateral", C.c_int),
                ("color", C.c_int), ("use_iir", C.c_int)]


def make_cfg(width, height, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, window=32,
             edge_aware=True, bilateral=False, color=False, use_iir=True) -> _Cfg:
    return _Cfg(int(width), int(height), float(fps), float(amp), float(f_low), float(f_high),
                int(window), int(bool(edge_aware)), int(bool(bilateral)), int(bool(color)),
                int(bool(use_iir)))


def build_oracle() -> str:
    """Compiles liboracle.so (gcc only, no reference sources needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def _avx512_host() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f in flags for f in ("avx512f", "avx512dq", "avx512cd", "avx512bw", "avx512vl"))


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = self.lib = C.CDLL(path)
        L.orc_levels.restype = C.c_int
        L.orc_positions.restype = C.c_long
        L.orc_subband_dims.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_u8_to_float.argtypes = [_u8p, C.c_long, _f32p]
        L.orc_float_to_u8.argtypes = [_f32p, C.c_long, _u8p]
        L.orc_gray.argtypes = [_f32p, C.c_long, _f32p]
        L.orc_ycbcr.argtypes = [_f32p, C.c_long, _f32p, _f32p, _f32p]
        L.orc_ycbcr_to_rgb.argtypes = [_f32p, _f32p, _f32p, C.c_long, _f32p]
        L.orc_dwt_forward.argtypes = [_f32p, C.c_int, C.c_int, _f32p, _f32p]
        L.orc_dwt_inverse.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p]
        L.orc_iir_design.argtypes = [C.c_float, C.c_float, C.c_float, _f32p, C.POINTER(C.c_int)]
        L.orc_iir_preseed.argtypes = [_f32p, C.c_int, _f32p, C.c_long, _f32p]
        L.orc_iir_step.argtypes = [_f32p, _f32p, C.c_long, _f32p, _f32p]
        L.orc_mag_sum.argtypes = [_f32p, C.c_long]
        L.orc_mag_sum.restype = C.c_float
        L.orc_threshold.argtypes = [_f32p, C.c_long, C.c_int]
        L.orc_threshold.restype = C.c_float
        L.orc_amplify.argtypes = [_f32p, _f32p, C.c_float, C.c_float, C.c_int, C.c_int, _f32p]
        L.orc_fade_amp.argtypes = [C.c_float, C.c_int, C.c_int]
        L.orc_fade_amp.restype = C.c_float
        L.orc_box.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int]
        L.orc_guided.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_float]
        L.orc_gauss5.argtypes = [_f32p, _f32p, C.c_int, C.c_int]
        L.orc_gray_to_rgb.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_window_apply.argtypes = [_f32p, C.c_long, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_stream_new.argtypes = [C.POINTER(_Cfg)]
        L.orc_stream_new.restype = C.c_void_p
        L.orc_stream_free.argtypes = [C.c_void_p]
        L.orc_stream_process.argtypes = [C.c_void_p, _f32p, _f32p]
        L.orc_stream_batch.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
        L.orc_stream_get.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.orc_stream_get.restype = C.c_long
        L.orc_stream_frames_processed.argtypes = [C.c_void_p]

    # geometry
    def levels(self, w, h) -> int:
        return self.lib.orc_levels(w, h)

    def positions(self, w, h) -> int:
        return self.lib.orc_positions(w, h)

    def subband_dims(self, w, h):
        sw = (C.c_int * 4)()
        sh = (C.c_int * 4)()
        L = self.lib.orc_subband_dims(w, h, sw, sh)
        return [(sw[i], sh[i]) for i in range(L)]

    # stages
    def u8_to_float(self, u8: np.ndarray) -> np.ndarray:
        u8 = np.ascontiguousarray(u8, np.uint8)
        out = np.empty(u8.shape, np.float32)
        self.lib.orc_u8_to_float(u8.ravel(), u8.size, out.ravel())
        return out

    def float_to_u8(self, f: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(f, np.float32)
        out = np.empty(f.shape, np.uint8)
        self.lib.orc_float_to_u8(f.ravel(), f.size, out.ravel())
        return out

    def gray(self, rgb: np.ndarray) -> np.ndarray:
        rgb = np.ascontiguousarray(rgb, np.float32)
        n = rgb.size // 3
        y = np.empty(rgb.shape[:-1], np.float32)
        self.lib.orc_gray(rgb.ravel(), n, y.ravel())
        return y

    def ycbcr(self, rgb):
        rgb = np.ascontiguousarray(rgb, np.float32)
        n = rgb.size // 3
        out = [np.empty(rgb.shape[:-1], np.float32) for _ in range(3)]
        self.lib.orc_ycbcr(rgb.ravel(), n, *[o.ravel() for o in out])
        return out

    def ycbcr_to_rgb(self, y, cb, cr):
        n = y.size
        out = np.empty(y.shape + (3,), np.float32)
        self.lib.orc_ycbcr_to_rgb(*[np.ascontiguousarray(a, np.float32).ravel() for a in (y, cb, cr)],
                                  n, out.ravel())
        return out

    def dwt_forward(self, img: np.ndarray):
        h, w = img.shape
        dims = self.subband_dims(w, h)
        flat = np.empty(self.positions(w, h), np.float32)
        low = np.empty(dims[-1][0] * dims[-1][1], np.float32)
        self.lib.orc_dwt_forward(np.ascontiguousarray(img, np.float32).ravel(), w, h, flat, low)
        return flat, low

    def dwt_inverse(self, flat6, lowpass, w, h):
        img = np.empty((h, w), np.float32)
        self.lib.orc_dwt_inverse(np.ascontiguousarray(flat6, np.float32),
                                 np.ascontiguousarray(lowpass, np.float32), w, h, img.ravel())
        return img

    def iir_design(self, f_low, f_high, fs):
        c = np.empty(10, np.float32)
        wu = C.c_int()
        rc = self.lib.orc_iir_design(f_low, f_high, fs, c, C.byref(wu))
        return (c, wu.value) if rc == 0 else (None, -1)

    def iir_run(self, x: np.ndarray, f_low, f_high, fs, preseed=True):
        """x: [frames][n]; returns deltas [frames][n] (frame-by-frame)."""
        c, wu = self.iir_design(f_low, f_high, fs)
        x = np.ascontiguousarray(x, np.float32)
        F, n = x.shape
        st = np.zeros(4 * n, np.float32)
        if preseed:
            self.lib.orc_iir_preseed(c, wu, x[0], n, st)
        out = np.empty_like(x)
        for t in range(F):
            self.lib.orc_iir_step(c, x[t], n, st, out[t])
        return out

    def mag_sum(self, x) -> float:
        x = np.ascontiguousarray(x, np.float32)
        return self.lib.orc_mag_sum(x, x.size)

    def threshold(self, orig6, batch_form=False) -> float:
        x = np.ascontiguousarray(orig6, np.float32)
        return self.lib.orc_threshold(x, x.size, int(batch_form))

    def amplify(self, delta6, orig6, amp, thr, w, h):
        out = np.empty(len(orig6), np.float32)
        self.lib.orc_amplify(np.ascontiguousarray(delta6, np.float32),
                             np.ascontiguousarray(orig6, np.float32), amp, thr, w, h, out)
        return out

    def fade_amp(self, amp, frames_before, warmup) -> float:
        return self.lib.orc_fade_amp(amp, frames_before, warmup)

    def box(self, img, r=4):
        h, w = img.shape
        out = np.empty_like(img, dtype=np.float32)
        self.lib.orc_box(np.ascontiguousarray(img, np.float32).ravel(), out.ravel(), w, h, r)
        return out

    def guided(self, guide, p, r=4, eps=0.01):
        h, w = guide.shape
        out = np.empty((h, w), np.float32)
        self.lib.orc_guided(np.ascontiguousarray(guide, np.float32).ravel(),
                            np.ascontiguousarray(p, np.float32).ravel(), out.ravel(), w, h, r, eps)
        return out

    def gray_to_rgb(self, gray, rgb, edge_aware=True):
        h, w = gray.shape
        out = np.empty((h, w, 3), np.float32)
        self.lib.orc_gray_to_rgb(np.ascontiguousarray(gray, np.float32).ravel(),
                                 np.ascontiguousarray(rgb, np.float32).ravel(), w, h,
                                 int(edge_aware), out.ravel())
        return out

    def window_apply(self, ring, ws, head, bilateral):
        ring = np.ascontiguousarray(ring, np.float32)
        n = ring.size // ws
        out = np.empty(n, np.float32)
        self.lib.orc_window_apply(ring.ravel(), n, ws, head, int(bilateral), out)
        return out

    def stream(self, **cfg) -> "_Stream":
        return _Stream(self.lib, "orc", make_cfg(**cfg))


class _Stream:
    """One video stream through either the oracle or the reference harness."""

    def __init__(self, lib, prefix, cfg: _Cfg, batch_size=0, threads=0):
        self.lib, self.cfg, self.p = lib, cfg, prefix
        if prefix == "orc":
            self.h = lib.orc_stream_new(C.byref(cfg))
        else:
            self.h = lib.rh_stream_new(C.byref(cfg), batch_size, threads)
        if not self.h:
            raise ValueError("stream init failed (invalid parameters)")
        self.P = cfg.width * cfg.height

    def process(self, rgb: np.ndarray) -> np.ndarray:
        rgb = np.ascontiguousarray(rgb, np.float32)
        out = np.empty_like(rgb)
        getattr(self.lib, f"{self.p}_stream_process")(self.h, rgb.ravel(), out.ravel())
        return out

    def batch(self, frames: np.ndarray) -> np.ndarray:
        frames = np.ascontiguousarray(frames, np.float32)
        out = np.empty_like(frames)
        fn = self.lib.orc_stream_batch if self.p == "orc" else self.lib.rh_batch_process
        n = fn(self.h, frames.ravel(), out.ravel(), frames.shape[0])
        if n != frames.shape[0]:
            raise RuntimeError("batch processing failed")
        return out

    def get(self, what: int, n: int) -> np.ndarray:
        buf = np.empty(n, np.float32)
        got = getattr(self.lib, f"{self.p}_stream_get")(self.h, what, buf)
        if got < 0:
            raise KeyError(what)
        return buf[:got]

    def close(self):
        if self.h:
            getattr(self.lib, f"{self.p}_stream_free")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Reference:
    """The reference library (compiled from its own sources) via ref_harness."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO) and _avx512_host()

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        if not _avx512_host():
            raise OSError("the reference build uses AVX-512; this host lacks it")
        L = self.lib = C.CDLL(path)
        L.rh_levels.restype = C.c_int
        L.rh_num_positions.restype = C.c_long
        L.rh_gray.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.rh_dwt_forward.argtypes = [_f32p, C.c_int, C.c_int, _f32p, _f32p]
        L.rh_dwt_inverse.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p]
        L.rh_coeff_amplify.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p]
        L.rh_iir_design.argtypes = [C.c_float, C.c_float, C.c_float, _f32p, C.POINTER(C.c_int)]
        L.rh_iir_run.argtypes = [_f32p, C.c_long, C.c_int, C.c_float, C.c_float, C.c_float,
                                 C.c_int, C.c_int, _f32p]
        L.rh_gray_to_rgb.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.rh_stream_new.argtypes = [C.POINTER(_Cfg), C.c_int, C.c_int]
        L.rh_stream_new.restype = C.c_void_p
        L.rh_stream_free.argtypes = [C.c_void_p]
        L.rh_stream_process.argtypes = [C.c_void_p, _f32p, _f32p]
        L.rh_batch_process.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
        L.rh_stream_get.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.rh_stream_get.restype = C.c_long
        L.rh_set_threads.argtypes = [C.c_int]
        L.rh_set_threads.restype = C.c_int

    def set_threads(self, n: int) -> int:
        return self.lib.rh_set_threads(n)

    def gray(self, rgb):
        h, w = rgb.shape[:2]
        y = np.empty((h, w), np.float32)
        self.lib.rh_gray(np.ascontiguousarray(rgb, np.float32).ravel(), w, h, y.ravel())
        return y

    def dwt_forward(self, img):
        h, w = img.shape
        n = self.lib.rh_num_positions(w, h)
        flat = np.empty(n, np.float32)
        low = np.empty(w * h, np.float32)
        self.lib.rh_dwt_forward(np.ascontiguousarray(img, np.float32).ravel(), w, h, flat, low)
        L = self.lib.rh_levels(w, h)
        lw, lh = w, h
        for _ in range(L):
            lw, lh = (lw + 1) // 2, (lh + 1) // 2
        return flat, low[:lw * lh].copy()

    def dwt_inverse(self, flat6, lowpass, w, h):
        img = np.empty((h, w), np.float32)
        self.lib.rh_dwt_inverse(np.ascontiguousarray(flat6, np.float32),
                                np.ascontiguousarray(lowpass, np.float32), w, h, img.ravel())
        return img

    def coeff_amplify(self, delta6, orig6, alpha, w, h):
        out = np.empty(len(orig6), np.float32)
        self.lib.rh_coeff_amplify(np.ascontiguousarray(delta6, np.float32),
                                  np.ascontiguousarray(orig6, np.float32), alpha, w, h, out)
        return out

    def iir_design(self, f_low, f_high, fs):
        c = np.empty(10, np.float32)
        wu = C.c_int()
        rc = self.lib.rh_iir_design(f_low, f_high, fs, c, C.byref(wu))
        return (c, wu.value) if rc == 0 else (None, -1)

    def iir_run(self, x, f_low, f_high, fs, preseed=True, batch=False):
        x = np.ascontiguousarray(x, np.float32)
        F, n = x.shape
        out = np.empty_like(x)
        rc = self.lib.rh_iir_run(x.ravel(), n, F, f_low, f_high, fs, int(preseed), int(batch),
                                 out.ravel())
        if rc != 0:
            raise ValueError("iir init failed")
        return out

    def gray_to_rgb(self, gray, rgb, edge_aware=True):
        h, w = gray.shape
        out = np.empty((h, w, 3), np.float32)
        self.lib.rh_gray_to_rgb(np.ascontiguousarray(gray, np.float32).ravel(),
                                np.ascontiguousarray(rgb, np.float32).ravel(), w, h,
                                int(edge_aware), out.ravel())
        return out

    def stream(self, batch_size=0, threads=0, **cfg) -> _Stream:
        return _Stream(self.lib, "rh", make_cfg(**cfg), batch_size, threads)
