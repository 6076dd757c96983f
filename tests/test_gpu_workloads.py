"""GPU parity on the benchmark workloads' own streams and settings, against the
oracle frame by frame, long enough to run through the reference's 15-frame
fade-in (wema.c:829-838, wema_batch.c:426-435) into full amplitude, where one
flipped threshold bit is worth tens of LSB:

* one stream of each size of the 48-stream mix (640x480, 1280x720,
  1920x1080 @ 60 fps, 3840x2160), with the mix's own seeds, discs, amps and
  0.5-5 Hz band, advanced together by batched ticks for 24 frames: every
  output within 1 LSB, every stream's threshold bit-exact on every frame;
* the 320x240 luma configuration (amp 50, 0.5-3 Hz) for its full 300 frames
  through the single-frame route, and for 64 frames through the batch route's
  threshold form (wema_batch.c:276): Y plane, all six coefficient slots,
  threshold, deltas, amplified coefficients and reconstructed Y bit-exact,
  output within 1 LSB;
* the 1920x1080 colour configuration (amp 120) for 24 frames: the three
  thresholds and the RGB24 output bit-exact;
* the 1280x720 @ 240 fps narrow band (0.2-0.6 Hz, amp 200, FP32), whose
  preseed runs 1336 cascade steps (iir_filter.c:376-471), for 24 frames:
  deltas and threshold bit-exact, output within 1 LSB.

The oracle runs every frame; the generator, oracle and device all start from
the same seeded u8 frames.
"""
import numpy as np
import pytest

from wema_b200 import cuda as wc
from wema_b200 import synth
from wema_b200.synth import SynthVideo

pytestmark = pytest.mark.gpu

FADE_FRAMES = 15


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def bits(x: float) -> int:
    return int(u32([x])[0])


def slot_mask(oracle, w, h, slots=(0, 1, 2)):
    m = []
    for (sw, sh) in oracle.subband_dims(w, h):
        for s in range(6):
            m.append(np.full(sw * sh, s in slots))
    return np.concatenate(m)


def lsb(a, b) -> np.ndarray:
    return np.abs(a.astype(np.int16) - b.astype(np.int16))


def mix_sample():
    """The first stream of each resolution of the 48-stream mix (seed 7)."""
    seen, out = set(), []
    for spec, cfg in synth.mixed_streams(seed=7):
        if (spec.width, spec.height) not in seen:
            seen.add((spec.width, spec.height))
            out.append((spec, cfg))
    return out


def test_mixed_workload_streams_against_oracle(oracle, torch_cuda):
    torch = torch_cuda
    F = 24
    sample = mix_sample()
    assert [(s.width, s.height) for s, _ in sample] == [(640, 480), (1280, 720), (1920, 1080),
                                                         (3840, 2160)]
    b = wc.Batch(device=0, max_streams=len(sample))
    ids, streams, inputs, outs, planes = [], [], [], [], []
    for spec, cfg in sample:
        w, h = spec.width, spec.height
        ids.append(b.add(w, h, **cfg))
        streams.append(oracle.stream(width=w, height=h, fps=cfg["fps"], amp=cfg["amp"],
                                     f_low=cfg["f_low"], f_high=cfg["f_high"],
                                     window=cfg["window"], edge_aware=True, color=False))
        inputs.append(SynthVideo(spec).frames(0, F))
        outs.append(torch.empty((h, w, 3), dtype=torch.uint8, device="cuda"))
        planes.append(oracle.positions(w, h))
    d_in = [torch.from_numpy(u).cuda() for u in inputs]
    worst = [0] * len(sample)
    for t in range(F):
        b.tick(ids, [d[t] for d in d_in], outs)
        b.sync()
        for k, (spec, cfg) in enumerate(sample):
            ref = oracle.float_to_u8(streams[k].process(oracle.u8_to_float(inputs[k][t])))
            d = lsb(ref, outs[k].cpu().numpy())
            worst[k] = max(worst[k], int(d.max()))
            assert d.max() <= 1, f"{spec.width}x{spec.height} frame {t}: {d.max()} LSB"
            orig = streams[k].get(2, planes[k])
            assert bits(b.threshold(ids[k])) == bits(oracle.threshold(orig)), \
                f"{spec.width}x{spec.height} frame {t}: threshold"
    assert F > FADE_FRAMES + 8
    b.close()


def _stream_pair(oracle, spec, **cfg):
    w, h = spec.width, spec.height
    so = oracle.stream(width=w, height=h, fps=spec.fps, **cfg)
    sg = wc.Session(width=w, height=h, fps=spec.fps, **cfg)
    return so, sg


def _check_planes(oracle, so, sg, w, h, m012, thr_form=0):
    N, P = len(m012), w * h
    assert np.array_equal(u32(sg.read(wc.READ_GRAY_IN)), u32(so.get(0, P))), "Y plane"
    orig = so.get(2, N)
    assert np.array_equal(u32(sg.read(wc.READ_ORIG6)), u32(orig)), "forward DWT"
    assert bits(sg.read(wc.READ_THRESHOLD)[0]) == bits(oracle.threshold(orig, thr_form)), "threshold"
    assert np.array_equal(u32(sg.read(wc.READ_DELTA6))[m012], u32(so.get(3, N))[m012]), "deltas"
    assert np.array_equal(u32(sg.read(wc.READ_AMP6))[m012], u32(so.get(4, N))[m012]), "amplified"
    assert np.array_equal(u32(sg.read(wc.READ_GRAY_OUT)), u32(so.get(1, P))), "inverse DWT"


def test_qvga_luma_configuration_300_frames(oracle, torch_cuda):
    torch = torch_cuda
    spec = synth.plain_qvga()
    w, h, F = spec.width, spec.height, 300
    u8 = SynthVideo(spec).frames(0, F)
    so, sg = _stream_pair(oracle, spec, amp=50.0, f_low=0.5, f_high=3.0, window=32,
                          edge_aware=True)
    m012 = slot_mask(oracle, w, h)
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    for t in range(F):
        ref = oracle.float_to_u8(so.process(oracle.u8_to_float(u8[t])))
        sg.process_u8(d_in[t], d_out)
        sg.sync()
        _check_planes(oracle, so, sg, w, h, m012)
        d = lsb(ref, d_out.cpu().numpy())
        assert d.max() <= 1, f"frame {t}: {d.max()} LSB"
    sg.close()


def test_qvga_luma_configuration_batch_route(oracle, torch_cuda):
    """The reference's batch route (wema_batch_process): threshold (0.2/N)*sum."""
    torch = torch_cuda
    spec = synth.plain_qvga(seed=5)
    w, h, F = spec.width, spec.height, 64
    u8 = SynthVideo(spec).frames(0, F)
    rgb = oracle.u8_to_float(u8)
    so = oracle.stream(width=w, height=h, fps=spec.fps, amp=50.0, f_low=0.5, f_high=3.0)
    sg = wc.Session(width=w, height=h, fps=spec.fps, amp=50.0, f_low=0.5, f_high=3.0,
                    threshold_form=wc.THR_BATCH)
    m012 = slot_mask(oracle, w, h)
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    for t in range(F):
        ref = oracle.float_to_u8(so.batch(rgb[t:t + 1]))[0]
        sg.process_u8(d_in[t], d_out)
        sg.sync()
        _check_planes(oracle, so, sg, w, h, m012, thr_form=1)
        d = lsb(ref, d_out.cpu().numpy())
        assert d.max() <= 1, f"frame {t}: {d.max()} LSB"
    sg.close()


def test_fullhd_colour_configuration(oracle, torch_cuda):
    torch = torch_cuda
    spec = synth.plain_fullhd()
    w, h, F = spec.width, spec.height, 24
    u8 = SynthVideo(spec).frames(0, F)
    so, sg = _stream_pair(oracle, spec, amp=120.0, f_low=0.5, f_high=3.0, window=32,
                          edge_aware=True, bilateral=True, color=True)
    N = oracle.positions(w, h)
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    for t in range(F):
        ref = oracle.float_to_u8(so.process(oracle.u8_to_float(u8[t])))
        sg.process_u8(d_in[t], d_out)
        sg.sync()
        thrs = sg.read(wc.READ_THRESHOLD)          # one per channel
        for ch, code in enumerate((2, 7, 8)):
            thr = thrs[ch]
            assert bits(thr) == bits(oracle.threshold(so.get(code, N))), f"frame {t} channel {ch}"
        assert np.array_equal(d_out.cpu().numpy(), ref), f"frame {t}: colour output"
    sg.close()


def test_720p_240fps_narrow_band_fp32(oracle, torch_cuda):
    torch = torch_cuda
    spec = synth.precision_720p()
    w, h, F = spec.width, spec.height, 24
    c, warmup = oracle.iir_design(0.2, 0.6, spec.fps)
    assert warmup == 1336
    u8 = SynthVideo(spec).frames(0, F)
    so, sg = _stream_pair(oracle, spec, amp=200.0, f_low=0.2, f_high=0.6, window=64,
                          edge_aware=True)
    m012 = slot_mask(oracle, w, h)
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    for t in range(F):
        ref = oracle.float_to_u8(so.process(oracle.u8_to_float(u8[t])))
        sg.process_u8(d_in[t], d_out)
        sg.sync()
        _check_planes(oracle, so, sg, w, h, m012)
        d = lsb(ref, d_out.cpu().numpy())
        assert d.max() <= 1, f"frame {t}: {d.max()} LSB"
    assert sg.frames_processed == warmup + F
    sg.close()
