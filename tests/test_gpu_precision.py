"""Precision variants against the FP64 re-evaluation (oracle/fp64.py).

The narrow low band at a high frame rate (0.2-0.6 Hz at 240 fps, poles at
radius 0.9963) is where the reference's FP32 biquad state drifts.  The FP64
state variant (wema_cuda_config.iir_state_fp64) must follow the FP64 cascade
to FP32 rounding of its output, and so must sit far closer to it than the
FP32 state does.  Both cascades are fed the same (GPU, FP32) coefficients, so
the comparison isolates the state precision.  A batched FP64-state stream must
also equal the same stream alone, bit for bit.  In window mode the FP16 ring
variant (wema_cuda_config.ring_fp16) must stay within FP16 rounding of the
FP64 window filter over the same coefficients."""
import numpy as np
import pytest

import fp64
from wema_b200 import cuda as wc
from wema_b200.synth import SynthSpec, SynthVideo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def unique_slots(flat6, dims):
    out, k6 = [], 0
    for (sw, sh) in dims:
        n = sw * sh
        out.append(flat6[k6: k6 + 3 * n])
        k6 += 6 * n
    return np.concatenate(out).astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_fp64_state_follows_fp64_cascade(oracle, torch_cuda):
    torch = torch_cuda
    w, h, F = 320, 180, 48
    band = dict(fps=240.0, amp=200.0, f_low=0.2, f_high=0.6)
    spec = SynthSpec(w, h, 240.0, 3, [0.4], [0.15], 30.0, 3.0)
    u8 = SynthVideo(spec).frames(0, F)
    d_in = torch.from_numpy(u8).cuda()
    dims = oracle.subband_dims(w, h)
    c32, _ = oracle.iir_design(0.2, 0.6, 240.0)
    sess = {v: wc.Session(width=w, height=h, state_fp64=v, **band) for v in (False, True)}
    ref = fp64.Stream64(w, h, coef=c32, **band)
    err = {False: [], True: []}
    for t in range(F):
        o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        coef = None
        for v, s in sess.items():
            s.process_u8(d_in[t], o)
            torch.cuda.synchronize()
            c = unique_slots(s.read(wc.READ_ORIG6), dims)
            if coef is None:
                coef = c
            assert np.array_equal(c, coef)                  # same forward transform
            d = unique_slots(s.read(wc.READ_DELTA6), dims)
            err[v].append(d)
        d64 = ref.step(coef)                                 # FP64 cascade, same inputs
        err[False][-1] = rel(err[False][-1], d64)
        err[True][-1] = rel(err[True][-1], d64)
    e32, e64 = max(err[False]), max(err[True])
    assert e64 < 1e-6, f"FP64 state: rel L2 {e64:.2e}"     # one FP32 rounding of the output
    assert e64 * 10 < e32, f"FP64 state {e64:.2e} vs FP32 state {e32:.2e}"
    for s in sess.values():
        s.close()


def test_fp64_state_batched_equals_alone(torch_cuda):
    torch = torch_cuda
    F = 5
    cfgs = [(160, 96, dict(fps=240.0, amp=200.0, f_low=0.2, f_high=0.6, state_fp64=True)),
            (128, 80, dict(fps=30.0, amp=50.0))]
    data = [SynthVideo(SynthSpec(w, h, c["fps"], 7 + k, [0.5], [0.3], 12.0, 2.0)).frames(0, F)
            for k, (w, h, c) in enumerate(cfgs)]
    b = wc.Batch(device=0, max_streams=4)
    ids = [b.add(w, h, **c) for (w, h, c) in cfgs]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    outs = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)] for (w, h, _) in cfgs]
    for t in range(F):
        b.tick(ids, [d[t] for d in d_in], [o[t] for o in outs])
    b.sync()
    for k, (w, h, c) in enumerate(cfgs):
        s = wc.Session(width=w, height=h, **c)
        for t in range(F):
            o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
            s.process_u8(d_in[k][t], o)
            torch.cuda.synchronize()
            assert np.array_equal(o.cpu().numpy(), outs[k][t].cpu().numpy()), f"stream {k} frame {t}"
        s.close()
    b.close()


@pytest.mark.parametrize("bilateral", [False, True])
def test_fp16_ring_against_fp64_window(oracle, torch_cuda, bilateral):
    torch = torch_cuda
    w, h, ws = 160, 96, 16
    F = ws + 6
    cfg = dict(fps=30.0, amp=60.0, use_iir=False, window=ws, bilateral=bilateral)
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 5, [1.3], [0.4], 14.0, 2.0)).frames(0, F)
    d_in = torch.from_numpy(u8).cuda()
    dims = oracle.subband_dims(w, h)
    sess = {v: wc.Session(width=w, height=h, ring_fp16=v, **cfg) for v in (False, True)}
    hist = []
    worst = {False: 0.0, True: 0.0}
    lsb = 0
    for t in range(F):
        outs = {}
        for v, s in sess.items():
            o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
            s.process_u8(d_in[t], o)
            torch.cuda.synchronize()
            outs[v] = o.cpu().numpy().astype(int)
            coef = unique_slots(s.read(wc.READ_ORIG6), dims)
        hist.append(coef)
        if t < ws - 1:
            assert np.array_equal(outs[True], u8[t])       # passthrough until the ring is full
            continue
        d64 = fp64.window_delta(np.stack(hist[-ws:]), bilateral)
        scale = np.linalg.norm(coef)
        for v, s in sess.items():
            d = unique_slots(s.read(wc.READ_DELTA6), dims)
            worst[v] = max(worst[v], float(np.linalg.norm(d - d64) / scale))
        lsb = max(lsb, int(np.abs(outs[True] - outs[False]).max()))
    assert worst[False] < 1e-6, f"FP32 ring {worst[False]:.2e}"
    assert worst[True] < 1e-3, f"FP16 ring {worst[True]:.2e}"    # FP16 rounds to 2^-11 relative
    assert lsb <= 2, f"FP16 vs FP32 ring output differs by {lsb} LSB"
    for s in sess.values():
        s.close()


@pytest.mark.parametrize("color", [False, True])
def test_fp16_planes_variant(oracle, torch_cuda, color):
    """The FP16-plane variant (wema_cuda_config.planes_fp16): coefficient and
    delta planes and the reconstructed frame stored in FP16, FP32 arithmetic
    (LL and coarser reconstructions FP32).
    Exact properties: level-0 coefficients are the FP32 path's rounded to
    FP16; the deltas are the reference's FP32 cascade (the oracle's, FP32
    state) run on the stored FP16 coefficients, rounded to FP16; the
    threshold is the FP64 sum of the FP16 coefficients (not the reference's
    bit-exact FP32 sum); a batched FP16-plane stream equals the same stream
    alone, bit for bit.  The output's distance from the FP32 path grows with
    the amplification (FP16 rounding of the coefficients is amplified like
    the motion); it is only checked loosely here and reported by the
    precision report."""
    torch = torch_cuda
    w, h, F = 320, 180, 20
    cfg = dict(fps=30.0, amp=80.0, f_low=0.5, f_high=3.0, color=color)
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 9, [1.1], [0.4], 20.0, 2.0)).frames(0, F)
    d_in = torch.from_numpy(u8).cuda()
    dims = oracle.subband_dims(w, h)
    s32 = wc.Session(width=w, height=h, **cfg)
    s16 = wc.Session(width=w, height=h, planes_fp16=True, **cfg)
    b = wc.Batch(device=0, max_streams=2)
    other = b.add(96, 80, amp=30.0)                       # a neighbour in every tick
    bid = b.add(w, h, planes_fp16=True, **cfg)
    dn = torch.from_numpy(SynthVideo(SynthSpec(96, 80, 30.0, 2, [1.0], [0.3], 10.0, 2.0)).frames(0, 1)).cuda()
    on = torch.empty((80, 96, 3), dtype=torch.uint8, device="cuda")
    c6_hist, d16_hist, diffs = [], [], []
    for t in range(F):
        o32 = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        o16, ob = torch.empty_like(o32), torch.empty_like(o32)
        s32.process_u8(d_in[t], o32)
        s16.process_u8(d_in[t], o16)
        b.tick([other, bid], [dn[0], d_in[t]], [on, ob])
        b.sync()
        torch.cuda.synchronize()
        c32 = unique_slots(s32.read(wc.READ_ORIG6), dims)
        c6 = s16.read(wc.READ_ORIG6)
        c16 = unique_slots(c6, dims)
        n0 = 3 * dims[0][0] * dims[0][1]                 # level 0: the FP32 coefficients rounded
        assert np.array_equal(c16[:n0], c32[:n0].astype(np.float16).astype(np.float64)), f"frame {t}"
        # the LL planes stay FP32: every level's coefficients are the FP32 ones rounded
        assert np.array_equal(c16, c32.astype(np.float16).astype(np.float64)), f"frame {t}: all levels"
        thr16, s6 = s16.read(wc.READ_THRESHOLD)[0], s16.read(wc.READ_MAGSUM)[0]
        want = 2.0 * np.abs(c16).sum()
        assert abs(s6 - want) <= 1e-6 * want, "FP16 threshold sum"
        assert abs(thr16 - 0.2 * want / (2 * c16.size)) <= 1e-6 * thr16, "FP16 threshold"
        c6_hist.append(c6.astype(np.float32))
        d16_hist.append(unique_slots(s16.read(wc.READ_DELTA6), dims))
        g16 = o16.cpu().numpy()
        assert np.array_equal(ob.cpu().numpy(), g16), f"frame {t}: batched FP16 stream"
        diffs.append(np.abs(g16.astype(int) - o32.cpu().numpy().astype(int)))
    # the reference's FP32 cascade on the FP16 coefficients, rounded to FP16
    dref = oracle.iir_run(np.stack(c6_hist), 0.5, 3.0, 30.0)
    for t in range(F):
        want = unique_slots(dref[t], dims).astype(np.float16).astype(np.float64)
        assert np.array_equal(d16_hist[t], want), f"frame {t}: FP16 deltas"
    d = np.stack(diffs)
    # a changed threshold flips amplification masks, each flip a local blob of
    # amp x delta: large but rare differences; the mean stays small
    assert d.mean() < 2.5, f"FP16 vs FP32 output: mean {d.mean():.3f} LSB"
    for x in (s32, s16):
        x.close()
    b.close()
