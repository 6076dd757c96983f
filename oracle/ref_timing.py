"""Timing of the reference's own CPU path on this host (test and benchmark
infrastructure: bench.py's CPU-baseline leg and its reference arm only).

The reference library is compiled from its own sources with its Makefile
flags (``oracle/_ref``, see ``oracle/Makefile``) and driven through its public
API by ``oracle/ref_harness.c``.  Its fastest route for an IIR luma stream is
``wema_batch_process`` (wema_batch.c:352-457): OpenMP over the frames of a
batch for the DWT, amplification, inverse DWT and guided filter, over the
positions for the IIR.  A stream's first batch also runs
``iir_temporal_preseed`` (iir_filter.c:376-471, single-threaded, ``warmup``
cascade passes over frame 0), which is timed separately here and kept out of
the steady rate, as the device side's warm-up keeps its own preseed out.

Where the compiled reference is absent (or the host lacks AVX-512, which its
build targets), the oracle restatement (``oracle/wema_oracle.c``) is timed
instead, one frame at a time, and the result says ``kind: port``.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from oracle import Oracle, Reference

# frame memory the reference's batch route holds per pixel and frame: float
# RGB in and out (24 B), 6-slot coefficients, deltas and the DWT context
# (~8 B each over N6 ~ 2P positions), gray in / out (8 B)
BATCH_BYTES_PER_PIXEL = 56
BATCH_MEMORY_CAP = 8 << 30


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def batch_candidates(pixels: int, cores: int, sizes=(8, 16, 64)):
    """(batch, threads) pairs of the sweep: batch 8 / 16 / 64 x threads
    1 / all cores, batches whose frame memory exceeds the cap left out."""
    out = []
    for b in sizes:
        if b * pixels * BATCH_BYTES_PER_PIXEL > BATCH_MEMORY_CAP:
            continue
        for t in sorted({1, cores}):
            out.append((b, t))
    return out


def stream_cfg(width, height, cfg):
    return dict(width=width, height=height, fps=cfg["fps"], amp=cfg["amp"], f_low=cfg["f_low"],
                f_high=cfg["f_high"], window=cfg.get("window", 32),
                edge_aware=cfg.get("edge_aware", True), bilateral=cfg.get("bilateral", False),
                color=cfg.get("color", False), use_iir=True)


class RefStream:
    """One IIR luma stream through the reference's batch route."""

    def __init__(self, R: Reference, width, height, cfg, batch, threads):
        self.R, self.batch, self.threads = R, batch, threads
        self.P = width * height
        R.set_threads(threads)
        self.s = R.stream(batch_size=batch, threads=threads, **stream_cfg(width, height, cfg))

    def run(self, rgb: np.ndarray) -> float:
        """rgb: [n][h][w][3] float frames, n <= batch; returns seconds."""
        self.R.set_threads(self.threads)
        out = np.empty_like(rgb)
        fn = self.R.lib.rh_batch_process
        t0 = time.perf_counter()
        got = fn(self.s.h, rgb.ravel(), out.ravel(), rgb.shape[0])
        dt = time.perf_counter() - t0
        if got != rgb.shape[0]:
            raise RuntimeError("wema_batch_process returned %d of %d frames" % (got, rgb.shape[0]))
        return dt

    def close(self):
        self.s.close()


def preseed_ms(R: Reference, O: Oracle, rgb0: np.ndarray, cfg) -> float:
    """iir_temporal_preseed of one stream (init + warmup passes over frame 0's
    6-slot coefficients), single-threaded as in the reference."""
    h, w = rgb0.shape[:2]
    gray = R.gray(rgb0)
    flat, _ = R.dwt_forward(gray)
    n = flat.size
    out = np.empty(n, np.float32)
    t0 = time.perf_counter()
    rc = R.lib.rh_iir_run(flat, n, 0, cfg["f_low"], cfg["f_high"], cfg["fps"], 1, 0, out)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise ValueError("iir init failed")
    return dt * 1e3


def sweep_size(R, O, frames_u8, cfg, cores, frames_timed=16, log=None):
    """Every (batch, threads) candidate on one stream size: a 1-frame batch
    first (untimed: the preseed and first-touch allocation), then at least
    `frames_timed` steady frames in full batches.  Returns the candidates'
    rates and the best one."""
    F, h, w = frames_u8.shape[:3]
    rgb = O.u8_to_float(frames_u8)
    res = []
    for (b, t) in batch_candidates(w * h, cores):
        st = RefStream(R, w, h, cfg, b, t)
        st.run(rgb[:1])
        nb = max(1, -(-frames_timed // b))
        secs, nfr = 0.0, 0
        for i in range(nb):
            sl = rgb[np.arange(1 + i * b, 1 + (i + 1) * b) % F]
            secs += st.run(np.ascontiguousarray(sl))
            nfr += b
        st.close()
        r = w * h * nfr / secs / 1e6
        res.append({"batch": b, "threads": t, "frames": nfr, "mpix_frames_s": round(r, 3)})
        if log:
            log(f"reference {w}x{h} batch {b} threads {t}: {r:.2f} Mpix-frames/s")
    best = max(res, key=lambda x: x["mpix_frames_s"])
    return res, best


def mix_rate(per_size):
    """Aggregate Mpix-frames/s of a mix of stream sizes, each size's frames
    run at its own steady rate: per_size = [(streams, pixels, rate)]."""
    pix = sum(n * p for n, p, _ in per_size)
    secs = sum(n * p / (r * 1e6) for n, p, r in per_size)
    return pix / 1e6 / secs


def port_rate(O: Oracle, frames_u8, cfg, nframes):
    """The oracle restatement, one frame at a time after an untimed first
    frame (its preseed): Mpix-frames/s."""
    F, h, w = frames_u8.shape[:3]
    rgb = O.u8_to_float(frames_u8)
    s = O.stream(**stream_cfg(w, h, cfg))
    s.process(rgb[0])
    t0 = time.perf_counter()
    for t in range(nframes):
        s.process(rgb[(1 + t) % F])
    dt = time.perf_counter() - t0
    s.close()
    return w * h * nframes / dt / 1e6


def reference_available() -> bool:
    return Reference.available()
