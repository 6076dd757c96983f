"""Seeded synthetic RGB24 video (ctypes binding of ``synth/synth.c``).

The generator stands in for the lossless rawvideo/ffv1 inputs of the
benchmark workloads; every frame is a pure function of (params, index).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _build

MAX_DISCS = 4


class _Params(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fps", C.c_float),
                ("seed", C.c_uint64), ("n_discs", C.c_int),
                ("disc_freq", C.c_float * MAX_DISCS), ("disc_amp", C.c_float * MAX_DISCS),
                ("disc_radius", C.c_float), ("noise_sigma", C.c_float),
                ("flicker_amp", C.c_float), ("flicker_freq", C.c_float)]


@dataclass
class SynthSpec:
    width: int
    height: int
    fps: float = 30.0
    seed: int = 1
    disc_freq: list = field(default_factory=lambda: [1.2])
    disc_amp: list = field(default_factory=lambda: [0.3])
    disc_radius: float = 30.0
    noise_sigma: float = 2.0
    flicker_amp: float = 0.0
    flicker_freq: float = 0.1


_lib = None


def _load():
    global _lib
    if _lib is None:
        path = _build.synth_lib_path()
        if not os.path.exists(path):
            _build.build_synth()
        L = C.CDLL(path)
        L.synth_new.argtypes = [C.POINTER(_Params)]
        L.synth_new.restype = C.c_void_p
        L.synth_free.argtypes = [C.c_void_p]
        L.synth_frame.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.synth_frames.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        _lib = L
    return _lib


class SynthVideo:
    def __init__(self, spec: SynthSpec):
        if len(spec.disc_freq) != len(spec.disc_amp) or len(spec.disc_freq) > MAX_DISCS:
            raise ValueError("disc_freq/disc_amp must have equal length <= 4")
        self.spec = spec
        p = _Params()
        p.width, p.height, p.fps, p.seed = spec.width, spec.height, spec.fps, spec.seed
        p.n_discs = len(spec.disc_freq)
        for i, (f, a) in enumerate(zip(spec.disc_freq, spec.disc_amp)):
            p.disc_freq[i], p.disc_amp[i] = f, a
        p.disc_radius, p.noise_sigma = spec.disc_radius, spec.noise_sigma
        p.flicker_amp, p.flicker_freq = spec.flicker_amp, spec.flicker_freq
        self._lib = _load()
        self._h = self._lib.synth_new(C.byref(p))
        if not self._h:
            raise ValueError("invalid synthetic video parameters")

    def frames(self, t0: int, count: int, out: np.ndarray | None = None) -> np.ndarray:
        s = self.spec
        if out is None:
            out = np.empty((count, s.height, s.width, 3), np.uint8)
        assert out.dtype == np.uint8 and out.flags.c_contiguous and out.size == count * s.height * s.width * 3
        self._lib.synth_frames(self._h, t0, count, out.ctypes.data)
        return out

    def frame(self, t: int) -> np.ndarray:
        return self.frames(t, 1)[0]

    def close(self):
        if self._h:
            self._lib.synth_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- the benchmark workloads' generators -----------------------------------

def plain_qvga(seed: int = 1) -> SynthSpec:
    """320x240 @30, one disc 1.2 Hz / 0.3 px, noise 2 LSB."""
    return SynthSpec(320, 240, 30.0, seed, [1.2], [0.3], 30.0, 2.0)


def plain_fullhd(seed: int = 2) -> SynthSpec:
    """1920x1080 @30, discs 0.8/1.5/2.5 Hz (0.2-0.5 px), +-1 LSB flicker 0.1 Hz."""
    return SynthSpec(1920, 1080, 30.0, seed, [0.8, 1.5, 2.5], [0.5, 0.35, 0.2], 30.0, 2.0,
                     flicker_amp=1.0, flicker_freq=0.1)


def precision_720p(seed: int = 3) -> SynthSpec:
    """1280x720 @240, one disc 0.4 Hz / 0.15 px, noise 3 LSB."""
    return SynthSpec(1280, 720, 240.0, seed, [0.4], [0.15], 30.0, 3.0)


def mixed_streams(seed: int = 7):
    """The 48-stream batched workload: (SynthSpec, stream settings) per stream.
    16 x 640x480@30, 16 x 1280x720@30, 12 x 1920x1080@60, 4 x 3840x2160@30;
    each stream its own seed, 1-3 discs at 0.5-4 Hz (0.2-0.5 px), amp 20-150,
    window 16-64 (recorded; the IIR filter does not use it), band 0.5-5 Hz,
    luma with the edge-aware guided filter, FP32."""
    rng = np.random.default_rng(seed)
    mix = [(640, 480, 30.0, 16), (1280, 720, 30.0, 16), (1920, 1080, 60.0, 12), (3840, 2160, 30.0, 4)]
    out = []
    k = 0
    for (w, h, fps, n) in mix:
        for _ in range(n):
            nd = int(rng.integers(1, 4))
            spec = SynthSpec(w, h, fps, seed=1000 + k,
                             disc_freq=[float(x) for x in rng.uniform(0.5, 4.0, nd)],
                             disc_amp=[float(x) for x in rng.uniform(0.2, 0.5, nd)],
                             disc_radius=30.0 * min(w, h) / 480.0, noise_sigma=2.0)
            cfg = dict(fps=fps, amp=float(rng.uniform(20.0, 150.0)), f_low=0.5, f_high=5.0,
                       window=int(rng.integers(16, 65)), color=False, edge_aware=True)
            out.append((spec, cfg))
            k += 1
    return out


SERVED_RES = [((640, 480), 0.40), ((1280, 720), 0.30), ((1920, 1080), 0.25), ((3840, 2160), 0.05)]


def served_sessions(seed: int = 11, horizon_s: float = 30.0, rate_per_s: float = 2.0,
                    len_s=(5.0, 60.0)):
    """The served workload's session list: a Poisson process of stream
    sessions (mean `rate_per_s` arrivals per second) with lengths log-uniform
    in `len_s`, resolution drawn from 480p 40% / 720p 30% / 1080p 25% /
    2160p 5%, 30 or 60 fps, contents and settings as the mixed workload.
    Arrivals start at -len_s[1] so the sessions alive at t = 0 are a draw
    from the steady state; each is returned with its open time clipped to 0.
    Returns [(t_open, t_close, SynthSpec, settings)] for sessions alive in
    [0, horizon_s), ordered by open time."""
    rng = np.random.default_rng(seed)
    t = -float(len_s[1])
    out = []
    k = 0
    lo, hi = np.log(len_s[0]), np.log(len_s[1])
    while True:
        t += float(rng.exponential(1.0 / rate_per_s))
        if t >= horizon_s:
            break
        length = float(np.exp(rng.uniform(lo, hi)))
        ri = int(rng.choice(len(SERVED_RES), p=[p for _, p in SERVED_RES]))
        (w, h) = SERVED_RES[ri][0]
        fps = float(rng.choice([30.0, 60.0]))
        nd = int(rng.integers(1, 4))
        spec = SynthSpec(w, h, fps, seed=5000 + k,
                         disc_freq=[float(x) for x in rng.uniform(0.5, 4.0, nd)],
                         disc_amp=[float(x) for x in rng.uniform(0.2, 0.5, nd)],
                         disc_radius=30.0 * min(w, h) / 480.0, noise_sigma=2.0)
        cfg = dict(fps=fps, amp=float(rng.uniform(20.0, 150.0)), f_low=0.5, f_high=5.0,
                   window=int(rng.integers(16, 65)), color=False, edge_aware=True)
        k += 1
        if t + length <= 0.0:
            continue
        out.append((max(t, 0.0), min(t + length, horizon_s), spec, cfg))
    out.sort(key=lambda x: x[0])
    return out
