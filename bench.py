"""Benchmark: WEMA per-frame amplification on B200.

Workload (default, mixed_streams_48): 48 camera streams of uneven sizes
(16 x 640x480@30, 16 x 1280x720@30, 12 x 1920x1080@60, 4 x 3840x2160@30),
each with its own seed, 1-3 discs at 0.5-4 Hz, amp 20-150, IIR band 0.5-5 Hz,
luma with the edge-aware guided filter, FP32.  A step is one tick: one frame
of every stream through the batched path (one launch per kernel type over all
48 pyramids: RGB24 in -> forward DWT -> exact threshold -> IIR + amplify ->
inverse DWT -> guided filter -> RGB24 out).
* value: Mpix-frames/s of back-to-back ticks, inputs resident in HBM,
  device-timed with CUDA events.
* plain_gpu / batched_over_plain: the same frames through one session per
  stream, one stream at a time, each frame waited for.
* latency_ms: p50/p99 per-frame latency with ticks paced at 60 Hz (30 fps
  streams in every other tick).
* e2e: the same ticks with every frame copied in from pinned host memory
  and every output copied back.
* roofline: the dominant stage's algorithmic bytes per tick over its mean
  device time (events around each stage on its stream, a separate pass)
  against the measured HBM copy bandwidth.
* cpu_baseline: the reference's own C path (compiled from its sources with
  its Makefile flags, oracle/_ref) on this host, a bounded sample of the mix.

Other workloads (--workload): plain_fullhd_color (one 1920x1080 colour
stream, the reference's plain full-HD configuration), plain_fullhd_luma,
plain_qvga_luma, precision_720p_240fps, served_poisson (Poisson sessions
through the served request loop in real time) and precision_report (errors
of the precision variants against the FP64 re-evaluation).

Multi-GPU (torchrun): every rank runs independent streams (replicas; the
path has no cross-stream exchange), value = all ranks' pixels / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (synth factory, session kwargs)
    "plain_fullhd_color": ("plain_fullhd", dict(fps=30.0, amp=120.0, f_low=0.5, f_high=3.0,
                                                color=True, edge_aware=True, bilateral=True)),
    "plain_fullhd_luma": ("plain_fullhd", dict(fps=30.0, amp=120.0, f_low=0.5, f_high=3.0,
                                               color=False, edge_aware=True)),
    "plain_qvga_luma": ("plain_qvga", dict(fps=30.0, amp=50.0, f_low=0.5, f_high=3.0,
                                           color=False, edge_aware=True)),
    "precision_720p_240fps": ("precision_720p", dict(fps=240.0, amp=200.0, f_low=0.2,
                                                     f_high=0.6, color=False, edge_aware=True)),
    # 48 streams of uneven sizes advanced one frame per tick (wema_cuda_batch_*)
    "mixed_streams_48": ("mixed_streams", None),
    # Poisson stream sessions through the served request loop (wema_cuda_server_*)
    "served_poisson": ("served_sessions", None),
    # the 48 streams of the mix on the served loop, clients keeping their queues full
    "served_saturated": ("mixed_streams", None),
    # error report of the precision variants against the FP64 re-evaluation
    "precision_report": ("precision_720p", None),
    # a small batched case for full ncu captures: 8 x 640x480 + 8 x 1920x1080
    # streams of the mix, 6 ticks, each synchronised (not a benchmark line)
    "profile_batch16": ("mixed_streams", None),
}
METRIC = "Mpix-frames/s"

# DRAM bytes (read + written) per launch of a stage's kernels from ncu
# captures (summaries and commands in profiles/), keyed by (workload, stage);
# stages not captured report null.  The batched kernels were captured on a
# tick of 16 streams (8 x 640x480 + 8 x 1920x1080, 19.05 Mpix,
# `--workload profile_batch16`) and are scaled by pixels to the 77.72 Mpix of
# the 48-stream tick; the threshold of the plain workload is monoids + walk.
_MIX = 77.722 / 19.046
TRAFFIC_NCU = {
    ("mixed_streams_48", "fwd_dwt_level0"): int((288116224 + 304738048) * _MIX),
    ("mixed_streams_48", "luma_transfer"): int((148669184 + 34321152) * _MIX),
    ("mixed_streams_48", "inv_dwt_level0"): int((133352960 + 47001344) * _MIX),
    ("plain_fullhd_color", "threshold"): 25081088 + 2323456,
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed_streams_48", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-frames", type=int, default=12, help="reference frames timed on the host")
    ap.add_argument("--served-seconds", type=float, default=20.0, help="served_poisson measured window")
    ap.add_argument("--precision-frames", type=int, default=480, help="precision_report frames")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sweep", default="full", choices=["full", "none"],
                    help="reference arm: sweep batch x threads per size (full), or batch 16 / 8 on "
                         "all cores only (none)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # the sampler's start-up (NVML initialisation) before the timed region:
        # wait, at most 3 s, for its first sample
        t_end = time.time() + 3.0
        while self.proc and self.proc.poll() is None and time.time() < t_end \
                and os.path.getsize(self.path) == 0:
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def stage_bytes(w, h, channels, levels_dims, pu, fused=True):
    """Algorithmic HBM bytes per frame of each stage: every plane its stage
    reads or writes, once (the 6-slot mirror of the threshold is the same
    memory as the unique planes, so it is counted once).  fused: the IIR
    step runs inside the forward transform (every frame after a stream's
    first): its state in / out and delta out (36 B per coefficient) count
    with the forward stage of the coefficient's level, and the coefficient
    is not read again."""
    P = w * h
    C = channels
    n0 = levels_dims[0][0] * levels_dims[0][1]
    step = C * (32 + 4) * 3                            # per position of a level: 3 coefficients
    fwd0 = 3 * P + C * 4 * 4 * n0                      # RGB24 in; LL + 3 bands out
    if fused:
        fwd0 += step * n0
    rest = 0
    for l in range(1, len(levels_dims)):
        pw, ph = levels_dims[l - 1]
        sw, sh = levels_dims[l]
        rest += C * 4 * (pw * ph + 4 * sw * sh) + (step * sw * sh if fused else 0)
    thr = C * 4 * pu                                   # |x| of every unique coefficient
    temporal = 0 if fused else C * (4 + 32 + 4) * pu   # coef in, state in/out, delta out
    inv = {}
    for l in range(len(levels_dims)):
        sw, sh = levels_dims[l]
        iw = (w if l == 0 else levels_dims[l - 1][0])
        ih = (h if l == 0 else levels_dims[l - 1][1])
        b = C * 4 * sw * sh + C * 8 * 3 * sw * sh      # LL in; 3 bands: coef + delta in
        b += 3 * P if (l == 0 and C == 3) else C * 4 * iw * ih
        inv[l] = b
    xfer = 0 if C == 3 else 3 * P + 4 * P + 3 * P      # RGB in, Y in, RGB out
    return {"fwd_dwt_level0": fwd0, "fwd_dwt_levels": rest, "threshold": thr,
            "temporal_amplify": temporal,
            "inv_dwt_levels": sum(v for l, v in inv.items() if l > 0),
            "inv_dwt_level0": inv[0], "luma_transfer": xfer}


# kernels behind each stage of a batched tick (one launch per tick over every stream)
STAGE_KERNELS_MULTI = {
    "fwd_dwt_level0": "k_dwt_fwd_multi<1,1> (level 0, RGB in, with the IIR step)",
    "fwd_dwt_levels": "k_dwt_fwd_multi<1,0> x 3 (with the IIR step)",
    "threshold": "k_thr_monoids_multi + k_thr_walk_multi",
    "temporal_amplify": "k_iir_multi (first frames only; else inside the forward transform)",
    "inv_dwt_levels": "k_dwt_inv_multi<1,0> x 3",
    "inv_dwt_level0": "k_dwt_inv_multi<1,0> (level 0)",
    "luma_transfer": "k_guided_transfer_multi",
}

# kernels behind each stage (one launch per frame unless noted)
STAGE_KERNELS = {
    "fwd_dwt_level0": "k_dwt_fwd<1|2> (level 0, RGB in)",
    "fwd_dwt_levels": "k_dwt_fwd<0> x (levels - 1)",
    "threshold": "k_thr_monoids + k_thr_walk",
    "temporal_amplify": "k_iir x channels",
    "inv_dwt_levels": "k_dwt_inv<1,0> x (levels - 1)",
    "inv_dwt_level0": "k_dwt_inv<3,1> (colour, RGB out) / k_dwt_inv<1,0> (luma)",
    "luma_transfer": "k_guided_transfer / k_gauss_transfer",
}


def dims_of(w, h):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    L = 0
    m = min(w, h)
    while m >= 16 and L < 4:
        m //= 2
        L += 1
    L = max(L, 1)
    dims = []
    for _ in range(L):
        w, h = (w + 1) // 2, (h + 1) // 2
        dims.append((w, h))
    return dims


def cpu_reference_rate(name, frames_u8, kw, nframes):
    """The reference's C path on this host: Mpix-frames/s over nframes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, Reference
    O = Oracle()
    h, w = frames_u8.shape[1:3]
    cfg = dict(width=w, height=h, fps=kw["fps"], amp=kw["amp"], f_low=kw["f_low"],
               f_high=kw["f_high"], color=kw.get("color", False),
               edge_aware=kw.get("edge_aware", True), bilateral=kw.get("bilateral", False))
    rgb = O.u8_to_float(frames_u8[:nframes])
    if Reference.available():
        R = Reference()
        cores = os.cpu_count() or 1
        R.set_threads(cores)
        kind = "reference"
        if cfg["color"]:
            s = R.stream(**cfg)
            cores_used = 1      # wema_process_frame is single-threaded
            t0 = time.perf_counter()
            for t in range(nframes):
                s.process(rgb[t])
            dt = time.perf_counter() - t0
        else:
            s = R.stream(batch_size=nframes, threads=cores, **cfg)
            cores_used = cores
            t0 = time.perf_counter()
            s.batch(rgb)
            dt = time.perf_counter() - t0
    else:
        kind = "port"
        cores_used = 1
        s = O.stream(**cfg)
        t0 = time.perf_counter()
        for t in range(nframes):
            s.process(rgb[t])
        dt = time.perf_counter() - t0
    value = w * h * nframes / dt / 1e6
    return {"value": round(value, 4), "unit": METRIC, "cores": cores_used, "kind": kind,
            "sample": f"{nframes} frames of {name} ({w}x{h}), first-frame preseed included"}


def _mix_sizes():
    """The mix's sizes: (first stream of the size, its settings, streams of
    that size in the mix)."""
    from wema_b200 import synth as S
    picks, count = {}, {}
    for spec, cfg in S.mixed_streams(seed=7):
        key = (spec.width, spec.height)
        count[key] = count.get(key, 0) + 1
        picks.setdefault(key, (spec, cfg))
    return [(spec, cfg, count[k]) for k, (spec, cfg) in picks.items()]


def mixed_cpu_sample(log=None):
    """The reference's CPU path on a bounded sample of the mix (about 20 s):
    for one stream of each size, wema_batch_process on all host cores
    (batches of 16 frames, 8 at 3840x2160), an untimed 1-frame first batch
    (the preseed, timed on its own), then 16 steady frames.  The sizes' rates
    are combined in the mix's proportions."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_timing as RT
    from oracle import Oracle, Reference
    from wema_b200 import synth as S
    O = Oracle()
    cores = RT.host_cores()
    per, rates = {}, []
    kind = "reference" if RT.reference_available() else "port"
    R = Reference() if kind == "reference" else None
    for spec, cfg, n in _mix_sizes():
        w, h = spec.width, spec.height
        b = 8 if w * h > 4_000_000 else 16
        fr = S.SynthVideo(spec).frames(0, b + 1)
        if R is not None:
            pre = RT.preseed_ms(R, O, O.u8_to_float(fr[:1])[0], cfg)
            st = RT.RefStream(R, w, h, cfg, b, cores)
            st.run(O.u8_to_float(fr[:1]))
            rgb = O.u8_to_float(fr[1:])
            secs = sum(st.run(rgb) for _ in range(-(-16 // b)))
            st.close()
            r = w * h * b * (-(-16 // b)) / secs / 1e6
            per[f"{w}x{h}"] = {"batch": b, "threads": cores, "mpix_frames_s": round(r, 3),
                               "preseed_ms": round(pre, 1)}
        else:
            r = RT.port_rate(O, fr, cfg, 4)
            per[f"{w}x{h}"] = {"threads": 1, "mpix_frames_s": round(r, 3)}
        rates.append((n, w * h, r))
    return {"value": round(RT.mix_rate(rates), 4), "unit": METRIC,
            "cores": cores if kind == "reference" else 1, "kind": kind,
            "sample": "one stream of each size of the mix: wema_batch_process, all cores, "
                      "batch 16 (8 at 3840x2160), 16 steady frames after an untimed first "
                      "batch; preseed timed separately; sizes combined in the mix's proportions",
            "per_size": per}


def reference_mixed(a):
    """The reference arm on the mixed workload: the reference's own C path
    (oracle/_ref) on this host's cores, like for like with the device's steady
    ticks.  Per size of the mix (one stream of each): the sweep of batch
    8 / 16 / 64 x threads 1 / all cores (each candidate an untimed 1-frame
    batch with the preseed, then >= 16 steady frames), the best candidate
    kept; its preseed time is reported on its own.  Then the timed steps:
    step i is one batch of size (i mod 4) through its best candidate, after
    `warmup` untimed steps; value = the sizes' steady rates combined in the
    mix's proportions (16 / 16 / 12 / 4 streams)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_timing as RT
    from oracle import Oracle, Reference
    from wema_b200 import synth as S
    O = Oracle()
    cores = RT.host_cores()
    sizes = _mix_sizes()
    K = max(1, min(a.steps, 40))
    W = a.warmup
    if not RT.reference_available():
        rates, per = [], {}
        for spec, cfg, n in sizes:
            fr = S.SynthVideo(spec).frames(0, 5)
            r = RT.port_rate(O, fr, cfg, 4)
            rates.append((n, spec.width * spec.height, r))
            per[f"{spec.width}x{spec.height}"] = {"threads": 1, "mpix_frames_s": round(r, 3)}
        v = RT.mix_rate(rates)
        return v, None, {"value": round(v, 4), "unit": METRIC, "cores": 1, "kind": "port",
                         "sample": "the oracle restatement, 4 frames per size", "per_size": per}
    R = Reference()
    log = (lambda m: print(m, file=sys.stderr, flush=True))
    per, rates, total_s, steps_done = {}, [], 0.0, 0
    for si, (spec, cfg, n) in enumerate(sizes):
        w, h = spec.width, spec.height
        bmax = max(b for b, _ in RT.batch_candidates(w * h, cores))
        fr = S.SynthVideo(spec).frames(0, bmax + 1)
        pre = RT.preseed_ms(R, O, O.u8_to_float(fr[:1])[0], cfg)
        if a.ref_sweep == "full":
            sweep, best = RT.sweep_size(R, O, fr, cfg, cores, log=log)
            b, t = best["batch"], best["threads"]
        else:
            sweep, b, t = [], (8 if w * h > 4_000_000 else 16), cores
        mine = [i for i in range(W + K) if i % len(sizes) == si]
        st = RT.RefStream(R, w, h, cfg, b, t)
        rgb = O.u8_to_float(fr)
        st.run(rgb[:1])
        secs, frames = 0.0, 0
        for i in mine:
            dt = st.run(np.ascontiguousarray(rgb[1:b + 1]))
            if i >= W:
                secs += dt
                frames += b
                steps_done += 1
        if frames == 0:                              # too few steps to reach this size
            secs = st.run(np.ascontiguousarray(rgb[1:b + 1]))
            frames = b
        st.close()
        total_s += secs
        r = w * h * frames / secs / 1e6
        rates.append((n, w * h, r))
        per[f"{w}x{h}"] = {"streams_in_mix": n, "batch": b, "threads": t,
                           "mpix_frames_s": round(r, 3), "frames_timed": frames,
                           "preseed_ms": round(pre, 1), "sweep": sweep}
    v = RT.mix_rate(rates)
    cb = {"value": round(v, 4), "unit": METRIC, "cores": cores, "kind": "reference",
          "sample": "one stream of each size of the mix through wema_batch_process; per size "
                    "the best of batch 8/16/64 x threads 1/all, steady frames after an "
                    "untimed first batch (preseed timed separately); sizes combined in the "
                    "mix's proportions",
          "per_size": per}
    return v, (total_s * 1e3 / max(steps_done, 1), steps_done), cb


DEFAULT_GROUPS = 1                         # the library's pipeline groups per steady tick


def mixed_config(world):
    from wema_b200 import synth as S
    pix = sum(spec.width * spec.height for spec, _ in S.mixed_streams(seed=7))
    return {"workload": "mixed_streams_48", "streams": 48,
            "mix": "16x640x480@30, 16x1280x720@30, 12x1920x1080@60, 4x3840x2160@30",
            "mode": "IIR 0.5-5 Hz, luma, edge-aware guided filter",
            "mpix_per_tick": round(pix / 1e6, 3), "step": "one tick = one frame of every stream",
            "parallelism": f"replicas x{world}", "l2": "per-tick working set > 126 MB L2 (no flush)"}


def plain_path_seconds(mix, d_in, d_out, local, t_stream, rounds, barrier):
    """The plain one-stream-at-a-time GPU path: each stream's frame alone
    through its own session, one after another, each waited for; seconds for
    `rounds` frames of every stream (first frames, with the preseed, untimed)."""
    import torch
    from wema_b200 import cuda as wc
    torch.cuda.synchronize()
    sess = [wc.Session(width=spec.width, height=spec.height, device=local, inspect=False, **cfg)
            for spec, cfg in mix]
    K = d_in[0].shape[0]
    for k in range(len(mix)):
        sess[k].process_u8(d_in[k][0], d_out[k], stream=t_stream)
    torch.cuda.synchronize()
    barrier()
    tp0 = time.perf_counter()
    for i in range(rounds):
        for k in range(len(mix)):
            sess[k].process_u8(d_in[k][(i + 1) % K], d_out[k], stream=t_stream)
            t_stream.synchronize()
    plain_s = time.perf_counter() - tp0
    for s in sess:
        s.close()
    return plain_s


def bench_mixed(a, rank, world, local):
    """The 48-stream mix: batched ticks against the plain one-stream-at-a-time
    GPU path, plus per-frame latency with ticks paced at 60 Hz (30 fps streams
    join every other tick)."""
    import torch
    from wema_b200 import cuda as wc
    from wema_b200 import synth as S

    from wema_b200 import replicas
    torch.cuda.set_device(local)
    dist = replicas.init("nccl")                 # replicas: every rank its own 48 streams
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    _, tune_report = wc.autotune(local)          # the filter's positions per thread, this device
    mix = S.mixed_streams(seed=7 + rank)
    K = 4                                             # unique frames per stream, cycled
    host, d_in, d_out = [], [], []
    for spec, cfg in mix:
        h = torch.empty((K, spec.height, spec.width, 3), dtype=torch.uint8).pin_memory()
        S.SynthVideo(spec).frames(0, K, out=h.numpy())
        host.append(h)
        d_in.append(h.to(dev))
        d_out.append(torch.empty((spec.height, spec.width, 3), dtype=torch.uint8, device=dev))
    pix = [spec.width * spec.height for spec, _ in mix]
    n = len(mix)
    b = wc.Batch(device=local, max_streams=n)
    ids = [b.add(spec.width, spec.height, **cfg) for spec, cfg in mix]
    t_stream = torch.cuda.Stream(device=dev)

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(t_stream)
        return e

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def tick(i, sel=None):
        sel = range(n) if sel is None else sel
        b.tick([ids[k] for k in sel], [d_in[k][i % K] for k in sel], [d_out[k] for k in sel])

    for i in range(a.warmup):
        tick(i)
    b.sync()
    l0 = b.stats()["launches"]
    barrier()
    with ClockSampler(local) as clk:
        e0, e1 = ev(), ev()
        e0.record(t_stream)
        b.tick([ids[0]], [d_in[0][0]], [d_out[0]], wait_event=e0)   # ordered after e0
        for i in range(a.steps):
            tick(a.warmup + i)
        b.tick([ids[0]], [d_in[0][1]], [d_out[0]], done_event=e1)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    launches = b.stats()["launches"] - l0
    clocks = clk.summary()
    barrier()
    frames_timed = a.steps * n + 2
    pix_timed = a.steps * sum(pix) + 2 * pix[0]

    # ---- the same ticks with the streams in 1..4 pipelined groups (the
    # library's default is the timed run above)
    groups_ms = {}
    for G in (1, 2, 3, 4):
        b.set_groups(G)
        for i in range(3):
            tick(i)
        b.sync()
        barrier()
        g0, g1 = ev(), ev()
        g0.record(t_stream)
        b.tick([ids[0]], [d_in[0][0]], [d_out[0]], wait_event=g0)
        for i in range(a.steps):
            tick(i)
        b.tick([ids[0]], [d_in[0][1]], [d_out[0]], done_event=g1)
        g1.synchronize()
        groups_ms[str(G)] = round(g0.elapsed_time(g1) / a.steps, 4)
    b.set_groups(DEFAULT_GROUPS)

    # ---- e2e through the host-frame tick (wema_cuda_batch_tick_host): every
    # tick's frames are copied in from pinned host memory and its outputs back,
    # double-buffered inside the library (tick i's outputs go out while tick
    # i+1's inputs come in and tick i runs).  A tick's 48 frames lie back to
    # back in one pinned arena (as a capture ring would hold them), so each
    # direction is one copy.  The host link carries 2 x 233 MB per tick and
    # bounds this.
    fb = [3 * p for p in pix]
    offs = np.concatenate([[0], np.cumsum(fb)]).astype(np.int64)
    arena_in = [torch.empty(int(offs[-1]), dtype=torch.uint8).pin_memory() for _ in range(K)]
    for i in range(K):
        for k in range(n):
            arena_in[i][offs[k]:offs[k + 1]].copy_(host[k][i].reshape(-1))
    arena_out = [torch.empty(int(offs[-1]), dtype=torch.uint8).pin_memory() for _ in range(2)]
    v_in = [[arena_in[i][offs[k]:offs[k + 1]] for k in range(n)] for i in range(K)]
    v_out = [[arena_out[j][offs[k]:offs[k + 1]] for k in range(n)] for j in range(2)]
    E = max(4, a.steps // 4)
    e2e_runs = {}
    for overlap in (False, True):               # True last: the library's default
        b.set_host_overlap(overlap)
        for i in range(3):                       # untimed: the library allocates its staging sets
            b.tick_host(ids, v_in[i % K], v_out[i % 2])
        b.sync()
        barrier()
        g0, g1 = ev(), ev()
        g0.record(t_stream)
        for i in range(E):
            b.tick_host(ids, v_in[i % K], v_out[i % 2],
                        wait_event=g0 if i == 0 else None, done_event=g1 if i == E - 1 else None)
        g1.synchronize()
        e2e_runs[overlap] = g0.elapsed_time(g1)
        barrier()
    e2e_ms = e2e_runs[True]

    # ---- latency at real rates: a tick every 1/60 s; the 60 fps streams take
    # part in every tick, the 30 fps ones in every other; latency of a frame =
    # its tick's submit-to-done time
    lat = []
    period = 1.0 / 60.0
    T = 60
    starts = [ev() for _ in range(T)]   # torch creates an event on its first record
    ends = [ev() for _ in range(T)]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(T):
        while time.perf_counter() < t0 + i * period:
            time.sleep(0.0002)
        sel = [k for k in range(n) if mix[k][1]["fps"] >= 60.0 or i % 2 == 0]
        starts[i].record(t_stream)
        b.tick([ids[k] for k in sel], [d_in[k][i % K] for k in sel], [d_out[k] for k in sel],
               wait_event=starts[i], done_event=ends[i])
        lat.append((i, len(sel)))
    ends[-1].synchronize()
    per_frame = []
    for (i, m) in lat:
        per_frame += [starts[i].elapsed_time(ends[i])] * m
    p50, p99 = float(np.percentile(per_frame, 50)), float(np.percentile(per_frame, 99))

    # ---- per-stage device time of the batched tick (a separate pass, so the
    # events do not touch the timed region; each tick alone, so a stage's time
    # is not stretched by the next tick's overlapping work)
    b.set_timing(True)
    for i in range(10):
        tick(i)
        b.sync()
    stage_tot, nt = b.stage_times()
    b.set_timing(False)
    per_tick = {k: v / max(nt, 1) for k, v in stage_tot.items()}
    sb = {}
    for spec, _ in mix:
        dims = dims_of(spec.width, spec.height)
        pu = sum(3 * sw * sh for sw, sh in dims)
        for k, v in stage_bytes(spec.width, spec.height, 1, dims, pu).items():
            sb[k] = sb.get(k, 0) + v
    peak, peak_kind = peaks()
    dom = max(per_tick, key=per_tick.get)
    achieved = sb[dom] / (per_tick[dom] * 1e-3) / 1e9
    total_bytes = sum(sb.values())
    roofline = {"bound": "hbm", "kernel": dom, "kernels": STAGE_KERNELS_MULTI[dom],
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": TRAFFIC_NCU.get(("mixed_streams_48", dom)),
                "algorithmic_bytes_per_launch": sb[dom]}
    pipeline = {"algorithmic_bytes_per_tick": total_bytes,
                "stage_ms_per_tick": {k: round(v, 4) for k, v in per_tick.items()},
                "stage_frac_of_hbm": {k: round(sb[k] / (per_tick[k] * 1e-3) / 1e9 / peak, 4)
                                      for k in per_tick if per_tick[k] > 0 and sb[k] > 0},
                "frac_of_hbm_roofline": round(total_bytes / (ms / a.steps * 1e-3) / 1e9 / peak, 4)}

    # ---- the plain one-stream-at-a-time GPU path
    b.close()
    P = max(2, a.steps // 8)
    plain_s = plain_path_seconds(mix, d_in, d_out, local, t_stream, P, barrier)

    if dist:
        t = torch.tensor([ms, e2e_ms, plain_s, p99], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms, plain_s, p99 = (float(x) for x in t)
    value = pix_timed * world / (ms * 1e-3) / 1e6
    plain = P * sum(pix) * world / plain_s / 1e6
    e2e = E * sum(pix) * world / (e2e_ms * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": mixed_config(world),
        "plain_gpu": {"value": round(plain, 2), "unit": METRIC,
                      "how": "each stream's frame through its own session, one at a time, waited for"},
        "batched_over_plain": round(value / plain, 3),
        "latency_ms": {"p50": round(p50, 3), "p99": round(p99, 3), "tick_hz": 60,
                       "frame_period_ms": {"60fps": 16.667, "30fps": 33.333}},
        "e2e": {"value": round(e2e, 2), "unit": METRIC, "h2d_bytes_per_step": 3 * sum(pix),
                "d2h_bytes_per_step": 3 * sum(pix),
                "how": "wema_cuda_batch_tick_host, host frames of a tick back to back in pinned memory "
                       "(one copy per direction), copies in beside the previous tick's kernels",
                "with_copies_in_after_the_previous_tick": round(E * sum(pix) * world / (e2e_runs[False] * 1e-3) / 1e6, 2)},
        "gpu_launches": launches, "frames_timed": frames_timed,
        "ms_per_step_by_pipeline_groups": groups_ms,
        "roofline": roofline, "pipeline": pipeline, "autotune": tune_report,
        "clocks": clocks,
    }
    if rank == 0 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = mixed_cpu_sample()
        except Exception as ex:   # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def bench_served(a, rank, world, local):
    """Stream sessions arriving as a Poisson process (2/s, lengths log-uniform
    5-60 s, the steady-state population open at t = 0) through the served
    request loop in real time; frames submitted at each stream's own rate.
    Reports completed Mpix-frames/s, per-frame latency and admission wait
    over the window after a warm-up."""
    import heapq
    import torch
    from wema_b200 import cuda as wc
    from wema_b200 import synth as S

    from wema_b200 import replicas
    torch.cuda.set_device(local)
    dist = replicas.init("nccl")                 # replicas: every rank serves its own sessions
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    warm, window = 3.0, float(a.served_seconds)
    horizon = warm + window
    sess = S.served_sessions(seed=11 + rank, horizon_s=horizon)
    K, R = 4, 12                                       # unique input frames per size; output ring
    inputs = {}
    for (_, _, spec, _) in sess:
        key = (spec.width, spec.height)
        if key not in inputs:
            h = torch.empty((K, spec.height, spec.width, 3), dtype=torch.uint8)
            S.SynthVideo(spec).frames(0, K, out=h.numpy())
            inputs[key] = h.to(dev)
    budget = 150 * 10**9
    srv = wc.Server(device=local, budget_bytes=budget, max_streams=512)
    rng = np.random.default_rng(5 + rank)
    ev = []                                            # (time, order, kind, session)
    for i, (t0, t1, _, _) in enumerate(sess):
        heapq.heappush(ev, (t0, 2 * i, "open", i))
        heapq.heappush(ev, (t1, 2 * i + 1, "close", i))
    sid, nfr, refused = {}, {}, 0
    # every session's output ring, allocated before the clock starts (clients own them)
    outs = {i: [torch.empty((spec.height, spec.width, 3), dtype=torch.uint8, device=dev)
                for _ in range(R)] for i, (_, _, spec, _) in enumerate(sess)}
    order = 2 * len(sess)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        reset_done = False
        while ev:
            t_ev = ev[0][0]
            now = time.perf_counter() - t_start
            if not reset_done and now >= warm:
                srv.stats(reset=True)
                reset_done = True
            if t_ev > now:
                time.sleep(min(t_ev - now, 0.0005))
                continue
            _, _, kind, i = heapq.heappop(ev)
            t0, t1, spec, cfg = sess[i]
            if kind == "open":
                sid[i] = srv.open(spec.width, spec.height, **cfg)
                nfr[i] = 0
                order += 1
                heapq.heappush(ev, (t0 + rng.uniform(0, 1.0 / cfg["fps"]), order, "frame", i))
            elif kind == "frame":
                if sid.get(i) is None:
                    continue
                k = nfr[i]
                rc = srv.submit(sid[i], inputs[(spec.width, spec.height)][k % K], outs[i][k % R])
                refused += rc != 0
                nfr[i] = k + 1
                t_next = t_ev + 1.0 / cfg["fps"]
                if t_next < t1:
                    order += 1
                    heapq.heappush(ev, (t_next, order, "frame", i))
            else:
                srv.close_session(sid[i])
                sid[i] = None
        st = srv.stats()
    srv.drain(120000)
    clocks = clk.summary()
    _, _, value = replicas.aggregate(st["mpix_frames"] * 1e6, st["seconds"] * 1e3, dist, device=dev)
    if dist:                                     # the worst rank's latencies
        t = torch.tensor([st["latency_p50_ms"], st["latency_p99_ms"], st["latency_max_ms"]],
                         dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        st["latency_p50_ms"], st["latency_p99_ms"], st["latency_max_ms"] = (float(x) for x in t)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC,
        "n_gpus": world, "steps": int(st["ticks"]), "warmup": 0,
        "ms_per_step": round(st["seconds"] * 1e3 / max(st["ticks"], 1), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "served_poisson", "arrivals_per_s": 2.0, "session_s": "log-uniform 5-60",
                   "mix": "480p 40%, 720p 30%, 1080p 25%, 2160p 5%; 30/60 fps",
                   "mode": "IIR 0.5-5 Hz, luma, edge-aware guided filter",
                   "window_s": window, "warmup_s": warm, "budget_bytes": budget,
                   "sessions": len(sess), "step": "one tick of the dispatcher",
                   "parallelism": f"replicas x{world}"},
        "frames": int(st["frames"]), "frames_refused": int(refused),
        "latency_ms": {"p50": round(st["latency_p50_ms"], 3), "p99": round(st["latency_p99_ms"], 3),
                       "max": round(st["latency_max_ms"], 3),
                       "frame_period_ms": {"60fps": 16.667, "30fps": 33.333}},
        "admission_wait_ms": {"p50": round(st["admission_wait_p50_ms"], 3),
                              "max": round(st["admission_wait_max_ms"], 3)},
        "sessions_admitted": int(st["sessions_admitted"]), "bytes_used_at_end": int(st["bytes_used"]),
        "dispatcher_ms": {k: round(st[k], 3) for k in ("tick_host_ms_mean", "tick_host_ms_max",
                                                       "tick_span_ms_mean", "tick_span_ms_max",
                                                       "admit_ms_max", "retire_ms_max")},
        "frames_per_tick": round(st["frames"] / max(st["ticks"], 1), 2),
        "gpu_launches": int(st["launches"]), "clocks": clocks,
    }
    srv.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def bench_served_saturated(a, rank, world, local):
    """The 48 streams of the mix opened on the served loop at once, every
    client keeping its queue full (it submits again whenever the server
    accepts), so frames arrive faster than ticks complete and each tick takes
    a frame of every live session: the served loop's saturated throughput
    against the plain one-stream-at-a-time GPU path, with per-frame latency
    (queueing included) and admission wait."""
    import torch
    from wema_b200 import cuda as wc
    from wema_b200 import synth as S

    from wema_b200 import replicas
    torch.cuda.set_device(local)
    dist = replicas.init("nccl")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mix = S.mixed_streams(seed=7 + rank)
    n, K, R = len(mix), 4, 16                  # unique inputs per stream; output ring (> 8 pending + 3 ticks)
    d_in, d_out, outs = [], [], []
    for spec, cfg in mix:
        h = torch.empty((K, spec.height, spec.width, 3), dtype=torch.uint8)
        S.SynthVideo(spec).frames(0, K, out=h.numpy())
        d_in.append(h.to(dev))
        d_out.append(torch.empty((spec.height, spec.width, 3), dtype=torch.uint8, device=dev))
        outs.append([torch.empty((spec.height, spec.width, 3), dtype=torch.uint8, device=dev)
                     for _ in range(R)])
    pix = [spec.width * spec.height for spec, _ in mix]
    budget = 150 * 10**9
    torch.cuda.synchronize(dev)
    srv = wc.Server(device=local, budget_bytes=budget, max_streams=64)
    sids = [srv.open(spec.width, spec.height, **cfg) for spec, cfg in mix]
    t_open = time.perf_counter()
    while any(srv.poll(x)["state"] != wc.SESSION_LIVE for x in sids):
        if time.perf_counter() - t_open > 60:
            raise RuntimeError("sessions not admitted within 60 s")
        time.sleep(0.001)
    admit_all_ms = (time.perf_counter() - t_open) * 1e3
    nfr = [0] * n
    warm, window = 1.0, min(float(a.served_seconds), 8.0)

    def pump(until):
        while time.perf_counter() < until:
            for k in range(n):
                # at most 8 pending + 3 ticks in flight per session: the ring of R outputs
                # is never overwritten while in use
                while srv.submit(sids[k], d_in[k][nfr[k] % K], outs[k][nfr[k] % R]) == 0:
                    nfr[k] += 1
            time.sleep(0.0002)

    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        pump(t0 + warm)
        srv.stats(reset=True)
        pump(time.perf_counter() + window)
        st = srv.stats()
    srv.drain(120000)
    clocks = clk.summary()
    srv.close()
    # the plain path on the same streams
    t_stream = torch.cuda.Stream(device=dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
    P = 4
    plain_s = plain_path_seconds(mix, d_in, d_out, local, t_stream, P, barrier)
    _, _, value = replicas.aggregate(st["mpix_frames"] * 1e6, st["seconds"] * 1e3, dist, device=dev)
    plain = P * sum(pix) * world / plain_s / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC,
        "n_gpus": world, "steps": int(st["ticks"]), "warmup": 0,
        "ms_per_step": round(st["seconds"] * 1e3 / max(st["ticks"], 1), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "served_saturated", "streams": n,
                   "mix": "16x640x480@30, 16x1280x720@30, 12x1920x1080@60, 4x3840x2160@30",
                   "mode": "IIR 0.5-5 Hz, luma, edge-aware guided filter",
                   "arrivals": "every client resubmits as soon as the server accepts (saturating)",
                   "window_s": window, "warmup_s": warm, "budget_bytes": budget,
                   "step": "one tick of the dispatcher", "parallelism": f"replicas x{world}"},
        "plain_gpu": {"value": round(plain, 2), "unit": METRIC,
                      "how": "each stream's frame through its own session, one at a time, waited for"},
        "served_over_plain": round(value / plain, 3),
        "frames": int(st["frames"]), "frames_per_tick": round(st["frames"] / max(st["ticks"], 1), 2),
        "latency_ms": {"p50": round(st["latency_p50_ms"], 3), "p99": round(st["latency_p99_ms"], 3),
                       "max": round(st["latency_max_ms"], 3),
                       "note": "submission to completion, queueing behind up to 8 pending frames included"},
        "admission": {"all_48_live_ms": round(admit_all_ms, 2),
                      "wait_p50_ms": round(st["admission_wait_p50_ms"], 3),
                      "wait_max_ms": round(st["admission_wait_max_ms"], 3)},
        "dispatcher_ms": {k: round(st[k], 3) for k in ("tick_host_ms_mean", "tick_host_ms_max",
                                                       "tick_span_ms_mean", "tick_span_ms_max",
                                                       "admit_ms_max")},
        "gpu_launches": int(st["launches"]), "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def _unique(flat6, dims):
    out, k6 = [], 0
    for (sw, sh) in dims:
        n = sw * sh
        out.append(flat6[k6: k6 + 3 * n])
        k6 += 6 * n
    return np.concatenate(out)


def bench_precision(a, rank, world, local):
    """Error report of the precision variants on the precision-stress stream
    (1280x720 @240 fps, one disc 0.4 Hz / 0.15 px, noise 3 LSB, band
    0.2-0.6 Hz, amp 200).  IIR: FP32 and FP64 biquad state, each frame's
    band-passed delta against the FP64 cascade fed the same coefficients, and
    the last frame's output against the FP64 pipeline (same threshold) and
    against the reference (its C restatement, bit-exact to it).  Window mode,
    ws 64: FP32 and FP16 ring, the last frame's delta against the FP64 window
    filter over the same coefficients (every 8th position), the output
    difference and the temporal stage's device time per frame."""
    if rank != 0:
        return
    import torch
    from wema_b200 import cuda as wc
    from wema_b200 import synth as S
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fp64
    from oracle import Oracle
    orc = Oracle()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    F = int(a.precision_frames)
    spec = S.precision_720p()
    w, h = spec.width, spec.height
    host = np.empty((F, h, w, 3), np.uint8)
    S.SynthVideo(spec).frames(0, F, out=host)
    d_in = torch.from_numpy(host).to(dev)
    dims = orc.subband_dims(w, h)
    band = dict(fps=240.0, amp=200.0, f_low=0.2, f_high=0.6)
    c32, warm = orc.iir_design(0.2, 0.6, 240.0)
    t0 = time.perf_counter()

    # ---- IIR: FP32 vs FP64 state
    # keys: False FP32 state, True FP64 state, "h16" FP16 planes (FP32 state)
    sess = {v: wc.Session(width=w, height=h, device=local, state_fp64=v, **band) for v in (False, True)}
    sess["h16"] = wc.Session(width=w, height=h, device=local, planes_fp16=True, **band)
    ref64 = fp64.Stream64(w, h, coef=c32, **band)
    rel = {False: [], True: [], "h16": []}
    absmax = {False: 0.0, True: 0.0, "h16": 0.0}
    outs = {}
    o = torch.empty((h, w, 3), dtype=torch.uint8, device=dev)
    coef = None
    for t in range(F):
        got = {}
        for v, s in sess.items():
            s.process_u8(d_in[t], o)
            torch.cuda.synchronize(dev)
            if v is False:
                coef = _unique(s.read(wc.READ_ORIG6), dims).astype(np.float64)
            got[v] = _unique(s.read(wc.READ_DELTA6), dims).astype(np.float64)
            if t == F - 1:
                outs[v] = o.cpu().numpy()
        d64 = ref64.step(coef)
        for v in sess:
            rel[v].append(float(np.linalg.norm(got[v] - d64) / np.linalg.norm(d64)))
            absmax[v] = max(absmax[v], float(np.abs(got[v] - d64).max()))
    thr = float(sess[False].read(wc.READ_THRESHOLD)[0])
    # the last frame through the FP64 pipeline: FP64 DWT, the FP64 delta, the same threshold
    flat, bands, low, I, rgb = ref64.coefficients(host[F - 1])
    amp = fp64.fade_amp(200.0, warm + F - 1, warm)
    nb, k = [], 0
    for l, lvl in enumerate(bands):
        al = amp * 0.5 if l == 0 else amp
        cur = []
        for b in lvl:
            dd = d64[k: k + b.size].reshape(b.shape)
            cur.append(np.where(np.abs(b) > thr, b + al * dd, b))
            k += b.size
        nb.append(tuple(cur))
    g64 = fp64.dwt_inverse(nb, low, w, h)
    out64 = fp64.to_u8(np.clip(rgb + fp64.guided(I, g64 - I)[..., None], 0.0, 1.0)).astype(int)
    so = orc.stream(width=w, height=h, **band)
    rgbf = orc.u8_to_float(host)
    for t in range(F):
        r = so.process(rgbf[t])
    out_ref = orc.float_to_u8(r).astype(int)

    def cmp(x, y):
        d = np.abs(x.astype(int) - y)
        return {"max_lsb": int(d.max()), "rms_lsb": round(float(np.sqrt((d.astype(float) ** 2).mean())), 5),
                "frac_gt1": float((d > 1).mean())}
    iir = {}
    for v, name in ((False, "fp32_state"), (True, "fp64_state"), ("h16", "fp16_planes")):
        iir[name] = {"state_bytes_per_position": 32 if v is True else 16,
                     "delta_rel_l2_vs_fp64": {"max": float(max(rel[v])), "last": rel[v][-1]},
                     "delta_max_abs_vs_fp64": absmax[v],
                     "output_vs_fp64": cmp(outs[v], out64), "output_vs_reference": cmp(outs[v], out_ref)}
    iir["fp16_planes"]["plane_bytes"] = "coefficient and delta planes and the reconstructed frame in FP16 (half the FP32 bytes)"
    iir["fp16_planes"]["output_vs_fp32_state"] = cmp(outs["h16"], outs[False].astype(int))
    for s in sess.values():
        s.close()

    # ---- window mode ws 64: FP32 vs FP16 ring
    ws = 64
    Fw = ws + 16
    wcfg = dict(fps=240.0, amp=200.0, use_iir=False, window=ws)
    ws_sess = {v: wc.Session(width=w, height=h, device=local, ring_fp16=v, **wcfg) for v in (False, True)}
    hist = []
    wouts = {}
    for t in range(Fw):
        for v, s in ws_sess.items():
            if t == ws:
                s.set_timing(True)
            s.process_u8(d_in[t % F], o)
            torch.cuda.synchronize(dev)
            if t == Fw - 1:
                wouts[v] = o.cpu().numpy()
        c = _unique(ws_sess[False].read(wc.READ_ORIG6), dims)
        hist.append(c[::8].copy())
    dw64 = fp64.window_delta(np.stack(hist[-ws:]), False)
    pu = sum(3 * sw * sh for (sw, sh) in dims)
    win = {}
    for v, name in ((False, "fp32_ring"), (True, "fp16_ring")):
        s = ws_sess[v]
        dv = _unique(s.read(wc.READ_DELTA6), dims)[::8].astype(np.float64)
        times, nfr = s.stage_times()
        ms = times["temporal_amplify"] / max(nfr, 1)
        win[name] = {"ring_bytes_per_frame": (ws + 1) * pu * (2 if v else 4),
                     "delta_rel_l2_vs_fp64": float(np.linalg.norm(dv - dw64) / np.linalg.norm(dw64)),
                     "temporal_stage_ms_per_frame": round(ms, 4)}
    win["fp16_ring"]["output_vs_fp32_ring"] = cmp(wouts[True], wouts[False].astype(int))
    for s in ws_sess.values():
        s.close()
    # ---- the plain 320x240 luma configuration (amp 50, 0.5-3 Hz, 300 frames):
    # every frame's output against the FP64 pipeline, with the GPU's threshold
    # (mask identical) and with the FP64 threshold (mask flips included)
    qs = S.plain_qvga(seed=1)
    qw, qh, QF = qs.width, qs.height, 300
    qu8 = S.SynthVideo(qs).frames(0, QF)
    qd = torch.from_numpy(qu8).to(dev)
    qcfg = dict(fps=30.0, amp=50.0, f_low=0.5, f_high=3.0)
    qsess = wc.Session(width=qw, height=qh, device=local, **qcfg)
    qc32, _ = orc.iir_design(0.5, 3.0, 30.0)
    q64 = {m: fp64.Stream64(qw, qh, coef=qc32, **qcfg) for m in ("gpu_thr", "fp64_thr")}
    qso = orc.stream(width=qw, height=qh, **qcfg)
    qrgb = orc.u8_to_float(qu8)
    acc = {m: [] for m in ("gpu_thr", "fp64_thr", "reference")}
    qo = torch.empty((qh, qw, 3), dtype=torch.uint8, device=dev)
    for t in range(QF):
        qsess.process_u8(qd[t], qo)
        torch.cuda.synchronize(dev)
        g = qo.cpu().numpy().astype(int)
        thr_t = float(qsess.read(wc.READ_THRESHOLD)[0])
        acc["gpu_thr"].append(np.abs(g - fp64.to_u8(q64["gpu_thr"].process(qu8[t], thr=thr_t)).astype(int)))
        acc["fp64_thr"].append(np.abs(g - fp64.to_u8(q64["fp64_thr"].process(qu8[t])).astype(int)))
        acc["reference"].append(np.abs(g - orc.float_to_u8(qso.process(qrgb[t])).astype(int)))
    qsess.close()
    qvga = {}
    for m, v in acc.items():
        d = np.stack(v)
        qvga[m] = {"max_lsb": int(d.max()), "rms_lsb": round(float(np.sqrt((d.astype(float) ** 2).mean())), 5),
                   "frac_gt1": float((d > 1).mean())}
    print(json.dumps({"metric": "precision", "workload": "precision_720p_240fps", "frames": F,
                      "config": {"size": f"{w}x{h}", "fps": 240, "band_hz": [0.2, 0.6], "amp": 200,
                                 "warmup": warm, "window": ws},
                      "iir": iir, "window_ws64": win,
                      "plain_qvga_luma_300_frames_output_error": {
                          "vs_fp64_same_threshold": qvga["gpu_thr"], "vs_fp64_own_threshold": qvga["fp64_thr"],
                          "vs_reference": qvga["reference"]},
                      "seconds": round(time.perf_counter() - t0, 1)}),
          flush=True)


def profile_batch16(a, rank, local):
    """6 synchronised ticks of 16 streams of the mix (the first 8 of 640x480
    and the first 8 of 1920x1080, seed 7): small enough for ncu --set full."""
    if rank != 0:
        return
    import torch
    from wema_b200 import cuda as wc
    from wema_b200 import synth as S
    torch.cuda.set_device(local)
    mall = S.mixed_streams(seed=7)
    mix = [m for m in mall if m[0].width == 640][:8] + [m for m in mall if m[0].width == 1920][:8]
    b = wc.Batch(device=local, max_streams=len(mix))
    ids, d_in, d_out = [], [], []
    for spec, cfg in mix:
        ids.append(b.add(spec.width, spec.height, **cfg))
        h = torch.empty((2, spec.height, spec.width, 3), dtype=torch.uint8)
        S.SynthVideo(spec).frames(0, 2, out=h.numpy())
        d_in.append(h.cuda())
        d_out.append(torch.empty((spec.height, spec.width, 3), dtype=torch.uint8, device="cuda"))
    for i in range(6):
        b.tick(ids, [d[i % 2] for d in d_in], d_out)
        b.sync()
    print(json.dumps({"workload": "profile_batch16", "streams": len(mix), "ticks": b.stats()["ticks"]}))
    b.close()


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    synth_name, kw = WORKLOADS[a.workload]
    if a.workload == "profile_batch16":
        return profile_batch16(a, rank, local)
    if a.workload == "precision_report":
        return bench_precision(a, rank, world, local)
    if a.workload == "served_saturated":
        if a.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no served "
                                  "form; its CPU path is timed on the mixed_streams_48 sample"}))
            return
        return bench_served_saturated(a, rank, world, local)
    if a.workload == "served_poisson":
        if a.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no served "
                                  "form; its CPU path is timed on the mixed_streams_48 sample"}))
            return
        return bench_served(a, rank, world, local)
    if a.workload == "mixed_streams_48":
        if a.impl != "reference":
            return bench_mixed(a, rank, world, local)
        if rank != 0:
            return
        v, timing, cb = reference_mixed(a)
        line = {"metric": METRIC, "value": round(v, 4), "unit": METRIC, "n_gpus": a.gpus,
                "steps": timing[1] if timing else 0, "warmup": a.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": mixed_config(a.gpus), "cpu_baseline": cb,
                "e2e": {"value": round(v, 4), "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        if timing:
            line["ms_per_step"] = round(timing[0], 3)
        print(json.dumps(line), flush=True)
        return

    from wema_b200 import synth as S
    spec = getattr(S, synth_name)(seed=1 + rank)
    w, h = spec.width, spec.height

    if a.impl == "reference":
        if rank != 0:
            return
        vid = S.SynthVideo(spec)
        nf = max(1, a.steps)
        frames = vid.frames(0, min(nf, 600))
        r = cpu_reference_rate(a.workload, frames, kw, min(nf, 600))
        line = {"metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": a.gpus,
                "steps": min(nf, 600), "warmup": 0, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": a.workload, "width": w, "height": h, "fps": kw["fps"]},
                "cpu_baseline": r,
                "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from wema_b200 import cuda as wc

    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    total = a.warmup + 3 * a.steps
    nuniq = min(600, max(total, 1))
    host = torch.empty((nuniq, h, w, 3), dtype=torch.uint8).pin_memory()
    S.SynthVideo(spec).frames(0, nuniq, out=host.numpy())
    d_frames = host.to(dev)
    d_out = torch.empty((h, w, 3), dtype=torch.uint8, device=dev)

    sess = wc.Session(width=w, height=h, device=local, inspect=False, **kw)
    t_stream = torch.cuda.Stream(device=dev)

    def frame(i):
        return d_frames[i % nuniq]

    def ev():
        # torch creates the CUDA event on its first record; the library then
        # re-records it on its own streams
        e = torch.cuda.Event(enable_timing=True)
        e.record(t_stream)
        return e

    # warm-up (includes the first frame's IIR preseed)
    for i in range(a.warmup):
        sess.process_u8(frame(i), d_out, stream=t_stream)
    torch.cuda.synchronize(dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- value: inputs resident in HBM; frames issued back to back (the
    # session overlaps frame t+1's forward transform and filter with frame
    # t's threshold and inverse); device time from an event the first frame
    # waits on to the event the last frame records
    k0 = a.warmup
    launches0 = sess.launches()
    barrier()
    with ClockSampler(local) as clk:
        ev0, ev1 = ev(), ev()
        ev0.record(t_stream)
        for i in range(a.steps):
            sess.process_u8_async(frame(k0 + i), d_out, wait_event=ev0 if i == 0 else None,
                                  done_event=ev1 if i == a.steps - 1 else None)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
    launches = sess.launches() - launches0
    barrier()
    clocks = clk.summary()

    # ---- per-stage timing pass: frames one at a time (each completes before
    # the next is issued), CUDA events around every stage on its own stream;
    # the threshold and the temporal filter of a frame still run side by side
    sess.set_timing(True)
    k1 = k0 + a.steps
    for i in range(a.steps):
        sess.process_u8(frame(k1 + i), d_out, stream=t_stream)
        torch.cuda.synchronize(dev)
    stages, nst = sess.stage_times()
    sess.set_timing(False)
    torch.cuda.synchronize(dev)

    # ---- e2e through the C ABI from pinned host frames: a ring of R device
    # buffers; H2D on one copy stream, D2H on another, each gated by the
    # library's per-frame done event
    k2 = k1 + a.steps
    R = 3
    d_in = [torch.empty((h, w, 3), dtype=torch.uint8, device=dev) for _ in range(R)]
    d_o = [torch.empty((h, w, 3), dtype=torch.uint8, device=dev) for _ in range(R)]
    h_out = torch.empty((R, h, w, 3), dtype=torch.uint8).pin_memory()
    s_h2d, s_d2h = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    ready = [ev() for _ in range(R)]
    done = [ev() for _ in range(R)]
    d2h_done = [ev() for _ in range(R)]
    barrier()
    e0, e1 = ev(), ev()
    e0.record(s_h2d)
    for i in range(a.steps):
        r = i % R
        with torch.cuda.stream(s_h2d):
            if i >= R:
                s_h2d.wait_event(done[r])        # input consumed
                s_h2d.wait_event(d2h_done[r])    # output read back
            d_in[r].copy_(host[(k2 + i) % nuniq], non_blocking=True)
            ready[r].record(s_h2d)
        sess.process_u8_async(d_in[r], d_o[r], wait_event=ready[r], done_event=done[r])
        with torch.cuda.stream(s_d2h):
            s_d2h.wait_event(done[r])
            h_out[r].copy_(d_o[r], non_blocking=True)
            d2h_done[r].record(s_d2h)
    e1.record(s_d2h)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    barrier()

    if dist:
        t = torch.tensor([ms, e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])

    pix = w * h
    value = pix * a.steps * world / (ms * 1e-3) / 1e6
    e2e = pix * a.steps * world / (e2e_ms * 1e-3) / 1e6

    dims = dims_of(w, h)
    pu = sum(3 * sw * sh for sw, sh in dims)
    C = 3 if kw.get("color") else 1
    sb = stage_bytes(w, h, C, dims, pu, fused=False)   # a plain session runs the IIR on its own
    per_frame = {k: v / max(nst, 1) for k, v in stages.items()}
    peak, peak_kind = peaks()
    dom = max(per_frame, key=per_frame.get)
    achieved = sb[dom] / (per_frame[dom] * 1e-3) / 1e9
    total_bytes = sum(sb.values())
    stage_frac = {k: round(sb[k] / (per_frame[k] * 1e-3) / 1e9 / peak, 4)
                  for k in per_frame if per_frame[k] > 0 and sb[k] > 0}
    traffic = TRAFFIC_NCU.get((a.workload, dom))

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": a.workload, "width": w, "height": h, "fps": kw["fps"],
                   "amp": kw["amp"], "band_hz": [kw["f_low"], kw["f_high"]],
                   "color": bool(kw.get("color")), "parallelism": f"replicas x{world}",
                   "l2": "per-frame working set > 126 MB L2 (no flush)"
                         if total_bytes > 126e6 else "working set fits L2 (no flush)"},
        "e2e": {"value": round(e2e, 2), "unit": METRIC, "h2d_bytes_per_step": 3 * pix,
                "d2h_bytes_per_step": 3 * pix},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "kernels": STAGE_KERNELS[dom],
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": sb[dom]},
        "pipeline": {"algorithmic_bytes_per_frame": total_bytes,
                     "stage_ms_per_frame": {k: round(v, 5) for k, v in per_frame.items()},
                     "stage_frac_of_hbm": stage_frac,
                     "frac_of_hbm_roofline": round(total_bytes / (ms / a.steps * 1e-3) / 1e9 / peak, 4)},
        "clocks": clocks,
    }
    if rank == 0 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_reference_rate(a.workload, host[:a.cpu_frames].numpy(), kw,
                                                      a.cpu_frames)
        except Exception as ex:   # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sess.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
