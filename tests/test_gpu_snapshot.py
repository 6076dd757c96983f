"""Snapshot / restore of a stream's state: a stream snapshotted after frame k
and restored into a fresh session (or batched stream) of the same config
continues exactly as the original - bit-identical frames - in IIR luma,
colour and window (bilateral) modes; a snapshot of another config is refused."""
import numpy as np
import pytest

from oracle_frames import assert_close, oracle_u8
from wema_b200 import cuda as wc
from wema_b200.synth import SynthSpec, SynthVideo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return torch


def run(torch, s, d, frames):
    outs = []
    for t in frames:
        o = torch.empty(d.shape[1:], dtype=torch.uint8, device="cuda")
        s.process_u8(d[t], o)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
    return outs


@pytest.mark.parametrize("cfg", [dict(amp=60.0), dict(amp=60.0, color=True),
                                 dict(amp=40.0, use_iir=False, window=8, bilateral=True)])
def test_session_snapshot_continues_exactly(oracle, torch_cuda, cfg):
    torch = torch_cuda
    w, h, F, K = 120, 88, 14, 9
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 13, [1.4], [0.4], 14.0, 2.0)).frames(0, F)
    d = torch.from_numpy(u8).cuda()
    a = wc.Session(width=w, height=h, fps=30.0, **cfg)
    run(torch, a, d, range(K))
    snap = a.snapshot()
    ref = run(torch, a, d, range(K, F))
    b = wc.Session(width=w, height=h, fps=30.0, **cfg)
    b.restore(snap)
    got = run(torch, b, d, range(K, F))
    want = oracle_u8(oracle, u8, fps=30.0, **cfg)
    for t in range(F - K):
        assert np.array_equal(got[t], ref[t]), f"frame {K + t}"
        assert_close(got[t], want[K + t], cfg.get("color", False), f"restored frame {K + t}")
    c = wc.Session(width=w + 8, height=h, fps=30.0, **cfg)
    with pytest.raises(RuntimeError):
        c.restore(snap)
    for s in (a, b, c):
        s.close()


def test_batched_stream_snapshot(oracle, torch_cuda):
    torch = torch_cuda
    w, h, F, K = 128, 96, 10, 6
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 21, [1.0], [0.4], 14.0, 2.0)).frames(0, F)
    d = torch.from_numpy(u8).cuda()
    o = [torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
    b1 = wc.Batch(device=0, max_streams=2)
    x = b1.add(w, h, amp=70.0)
    for t in range(K):
        b1.tick([x], [d[t]], [o[t]])
    snap = b1.snapshot(x)
    for t in range(K, F):
        b1.tick([x], [d[t]], [o[t]])
    b1.sync()
    ref = [o[t].cpu().numpy() for t in range(K, F)]
    b2 = wc.Batch(device=0, max_streams=2)
    other = b2.add(96, 80, amp=30.0)                 # a neighbour in the new batch
    y = b2.add(w, h, amp=70.0)
    b2.restore(y, snap)
    dn = torch.from_numpy(SynthVideo(SynthSpec(96, 80, 30.0, 5, [1.0], [0.3], 10.0, 2.0)).frames(0, 1)).cuda()
    on = torch.empty((80, 96, 3), dtype=torch.uint8, device="cuda")
    for t in range(K, F):
        b2.tick([other, y], [dn[0], d[t]], [on, o[t]])
    b2.sync()
    want = oracle_u8(oracle, u8, amp=70.0)
    for t in range(K, F):
        assert np.array_equal(o[t].cpu().numpy(), ref[t - K]), f"frame {t}"
        assert_close(o[t].cpu().numpy(), want[t], False, f"restored frame {t}")
    b1.close()
    b2.close()
