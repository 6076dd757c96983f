"""GPU parity: libwema_cuda (through its C ABI) against the oracle.

Bars (the oracle itself is pinned to the reference in test_oracle_pin.py):
  * bit-exact: Y / YCbCr planes, forward DWT coefficients (all six slots,
    including the reference's stale entries at odd level sizes), the
    threshold, IIR deltas and amplified coefficients of slots 0-2, the
    reconstructed Y, and the colour-mode output;
  * luma-mode output (guided filter / Gaussian): u8 within 1 LSB;
  * window mode deltas (reduction order and exp differ): relative L2 <= 1e-5,
    masks exact, u8 output within 1 LSB.
"""
import numpy as np
import pytest

from wema_b200 import cuda as wc
from wema_b200.synth import SynthSpec, SynthVideo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def slot_mask(oracle, w, h, slots=(0, 1, 2)):
    dims = oracle.subband_dims(w, h)
    m = []
    for (sw, sh) in dims:
        n = sw * sh
        for s in range(6):
            m.append(np.full(n, s in slots))
    return np.concatenate(m)


def frames_for(w, h, n, seed=3, fps=30.0):
    spec = SynthSpec(w, h, fps, seed, [1.3], [0.4], max(2.0, min(w, h) / 5), 2.0)
    return SynthVideo(spec).frames(0, n)


def run_pair(oracle, torch, w, h, F, **cfg):
    """Yields per frame (oracle stream, gpu session, oracle float out, gpu u8 out)."""
    u8 = frames_for(w, h, F, fps=cfg.get("fps", 30.0))
    rgb = oracle.u8_to_float(u8)
    ocfg = dict(width=w, height=h, fps=cfg.get("fps", 30.0), amp=cfg.get("amp", 50.0),
                f_low=cfg.get("f_low", 0.5), f_high=cfg.get("f_high", 3.0),
                window=cfg.get("window", 32), edge_aware=cfg.get("edge_aware", True),
                bilateral=cfg.get("bilateral", False), color=cfg.get("color", False),
                use_iir=cfg.get("use_iir", True))
    so = oracle.stream(**ocfg)
    sg = wc.Session(width=w, height=h, fps=ocfg["fps"], amp=ocfg["amp"], f_low=ocfg["f_low"],
                    f_high=ocfg["f_high"], window=ocfg["window"], edge_aware=ocfg["edge_aware"],
                    bilateral=ocfg["bilateral"], color=ocfg["color"], use_iir=ocfg["use_iir"])
    d_in = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    d_out = torch.empty_like(d_in)
    for t in range(F):
        o = so.process(rgb[t])
        d_in.copy_(torch.from_numpy(u8[t]))
        sg.process_u8(d_in, d_out)
        sg.sync()
        yield t, so, sg, o, d_out.cpu().numpy()


def check_frame(oracle, so, sg, o, g_u8, w, h, color, exact_out):
    N, P = oracle.positions(w, h), w * h
    m012 = slot_mask(oracle, w, h)
    assert np.array_equal(u32(sg.read(wc.READ_GRAY_IN)), u32(so.get(0, P))), "Y plane"
    orig_g, orig_o = sg.read(wc.READ_ORIG6), so.get(2, N)
    assert np.array_equal(u32(orig_g), u32(orig_o)), "forward DWT"
    assert np.array_equal(u32(sg.read(wc.READ_DELTA6))[m012], u32(so.get(3, N))[m012]), "deltas"
    assert np.array_equal(u32(sg.read(wc.READ_AMP6))[m012], u32(so.get(4, N))[m012]), "amplified"
    thr = sg.read(wc.READ_THRESHOLD)[0]
    assert u32([thr])[0] == u32([oracle.threshold(orig_o)])[0], "threshold"
    assert np.array_equal(u32(sg.read(wc.READ_GRAY_OUT)), u32(so.get(1, P))), "inverse DWT"
    q = oracle.float_to_u8(o)
    d = np.abs(q.astype(int) - g_u8.astype(int))
    if exact_out:
        assert d.max() == 0, "output"
    else:
        assert d.max() <= 1, f"output differs by {d.max()} LSB"
        assert (d > 0).mean() < 2e-3


@pytest.mark.parametrize("n", list(range(1, 41)) + [1000, 100003, 1 << 20, 4131360])
def test_threshold_flat_exact(oracle, torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    cases = [
        rng.standard_normal(n).astype(np.float32),
        (rng.standard_normal(n) * 10.0 ** rng.integers(-8, 4, n)).astype(np.float32),
        np.full(n, 0.1, np.float32),                       # ties galore
        (rng.integers(0, 4, n) * 2.0 ** -20).astype(np.float32),
        np.where(rng.random(n) < 0.5, 0.0, 1e-41).astype(np.float32),   # zeros and subnormals
    ]
    for x in cases:
        d = torch.from_numpy(x).cuda()
        for form in (0, 1):
            thr, s = wc.threshold_flat(d, form)
            assert u32([s])[0] == u32([oracle.mag_sum(x)])[0]
            assert u32([thr])[0] == u32([oracle.threshold(x, form)])[0]


@pytest.mark.parametrize("color", [False, True])
def test_stream_qvga(oracle, torch_cuda, color):
    w, h = 320, 240
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, 10, color=color, amp=50.0):
        check_frame(oracle, so, sg, o, g, w, h, color, exact_out=color)
        assert sg.frames_processed == so_frames(so)


def so_frames(so):
    return so.lib.orc_stream_frames_processed(so.h)


@pytest.mark.parametrize("w,h", [(136, 130), (240, 135), (37, 29), (17, 16), (64, 2), (3, 40),
                                 (100, 67), (1, 1), (33, 17)])
def test_stream_odd_sizes(oracle, torch_cuda, w, h):
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, 3, amp=80.0):
        check_frame(oracle, so, sg, o, g, w, h, False, exact_out=False)


def test_stream_odd_color(oracle, torch_cuda):
    w, h = 150, 133
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, 3, color=True, amp=120.0):
        check_frame(oracle, so, sg, o, g, w, h, True, exact_out=True)


def test_gaussian_fallback(oracle, torch_cuda):
    w, h = 200, 120
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, 3, edge_aware=False):
        check_frame(oracle, so, sg, o, g, w, h, False, exact_out=False)


@pytest.mark.parametrize("bilateral", [False, True])
@pytest.mark.parametrize("color", [False, True])
def test_window_mode(oracle, torch_cuda, bilateral, color):
    w, h, ws = 96, 80, 8
    N = oracle.positions(w, h)
    m012 = slot_mask(oracle, w, h)
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, ws + 4, use_iir=False, window=ws,
                                    bilateral=bilateral, color=color, amp=40.0):
        q = oracle.float_to_u8(o)
        assert np.abs(q.astype(int) - g.astype(int)).max() <= 1
        if t + 1 < ws:
            assert np.array_equal(q, g), "passthrough while the window fills"
            continue
        orig = so.get(2, N)
        assert np.array_equal(u32(sg.read(wc.READ_ORIG6)), u32(orig))
        dg, do = sg.read(wc.READ_DELTA6)[m012], so.get(3, N)[m012]
        rel = np.linalg.norm(dg.astype(np.float64) - do) / max(np.linalg.norm(do.astype(np.float64)), 1e-30)
        assert rel <= 1e-5
        thr = sg.read(wc.READ_THRESHOLD)[0]
        assert u32([thr])[0] == u32([oracle.threshold(orig)])[0]
        ag = sg.read(wc.READ_AMP6)[m012]
        mask_g = ag != orig[m012]
        mask_o = so.get(4, N)[m012] != orig[m012]
        assert np.array_equal(mask_g | (np.abs(orig[m012]) <= thr) , mask_o | (np.abs(orig[m012]) <= thr))


def test_batch_threshold_form(oracle, torch_cuda):
    torch = torch_cuda
    w, h, F = 160, 128, 6
    u8 = frames_for(w, h, F, seed=9)
    rgb = oracle.u8_to_float(u8)
    so = oracle.stream(width=w, height=h, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0)
    ref = oracle.float_to_u8(so.batch(rgb))
    sg = wc.Session(width=w, height=h, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0,
                    threshold_form=wc.THR_BATCH)
    for t in range(F):
        out = sg.process_host_u8(u8[t])
        assert np.abs(out.astype(int) - ref[t].astype(int)).max() <= 1


def test_float_input_path(oracle, torch_cuda):
    torch = torch_cuda
    w, h = 128, 96
    u8 = frames_for(w, h, 4, seed=5)
    rgb = oracle.u8_to_float(u8)
    a = wc.Session(width=w, height=h, fps=30.0, amp=60.0, f_low=0.5, f_high=3.0, color=True)
    b = wc.Session(width=w, height=h, fps=30.0, amp=60.0, f_low=0.5, f_high=3.0, color=True)
    so = oracle.stream(width=w, height=h, fps=30.0, amp=60.0, f_low=0.5, f_high=3.0, color=True)
    d_f = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    d_o = torch.empty_like(d_f)
    for t in range(4):
        d_f.copy_(torch.from_numpy(rgb[t]))
        a.process_f32(d_f, d_out_f32=d_o)
        a.sync()
        o = so.process(rgb[t])
        assert np.array_equal(u32(d_o.cpu().numpy()), u32(o)), "float path, colour: bit-exact"
        assert np.array_equal(b.process_host_u8(u8[t]), oracle.float_to_u8(o))


@pytest.mark.parametrize("color", [True, False])
def test_fullhd_frames(oracle, torch_cuda, color):
    """The 1920x1080 workload's geometry (odd 240x135 level-4 input, stale
    rows in the threshold) on its own seeded frames."""
    w, h = 1920, 1080
    for t, so, sg, o, g in run_pair(oracle, torch_cuda, w, h, 2, color=color, amp=120.0):
        check_frame(oracle, so, sg, o, g, w, h, color, exact_out=color)


def test_4k_threshold(oracle, torch_cuda):
    torch = torch_cuda
    w, h = 3840, 2160
    u8 = frames_for(w, h, 1, seed=12)
    y = oracle.gray(oracle.u8_to_float(u8)[0])
    orig, _ = oracle.dwt_forward(y)
    d = torch.from_numpy(orig).cuda()
    for form in (0, 1):
        thr, s = wc.threshold_flat(d, form)
        assert u32([thr])[0] == u32([oracle.threshold(orig, form)])[0]


@pytest.mark.parametrize("color", [False, True])
def test_pipelined_frames(oracle, torch_cuda, color):
    """Frames issued back to back without waiting (several in flight inside the
    session: forward/filter of frame t+1 overlap threshold/inverse of frame t)
    give the same outputs as the oracle run frame by frame."""
    torch = torch_cuda
    w, h, F = 256, 160, 12
    u8 = frames_for(w, h, F, seed=21)
    rgb = oracle.u8_to_float(u8)
    so = oracle.stream(width=w, height=h, fps=30.0, amp=90.0, f_low=0.5, f_high=3.0, color=color)
    ref = [oracle.float_to_u8(so.process(rgb[t])) for t in range(F)]
    sg = wc.Session(width=w, height=h, fps=30.0, amp=90.0, f_low=0.5, f_high=3.0, color=color,
                    inspect=False)
    d_in = torch.from_numpy(u8).cuda()
    outs = [torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
    torch.cuda.synchronize()
    for t in range(F):
        sg.process_u8_async(d_in[t], outs[t])
    sg.sync()
    for t in range(F):
        d = np.abs(outs[t].cpu().numpy().astype(int) - ref[t].astype(int))
        assert d.max() <= (0 if color else 1), f"frame {t}"
