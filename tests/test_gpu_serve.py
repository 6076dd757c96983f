"""The served request loop (wema_cuda_server_*): sessions that arrive while
others run are admitted and batched into the running ticks; every session's
frames equal the same stream run alone (bit-exact), however the sessions
overlapped; admission follows the device-memory budget first-in first-out."""
import time

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


def frames(w, h, n, seed, fps=30.0):
    spec = SynthSpec(w, h, fps, seed, [0.9 + 0.1 * seed], [0.4], max(2.0, min(w, h) / 5), 2.0)
    return SynthVideo(spec).frames(0, n)


def alone(torch, w, h, cfg, u8):
    s = wc.Session(width=w, height=h, **cfg)
    d_in = torch.from_numpy(u8).cuda()
    outs = []
    for t in range(u8.shape[0]):
        o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        s.process_u8(d_in[t], o)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
    s.close()
    return outs


def wait_for(pred, timeout=30.0):
    t0 = time.time()
    while not pred():
        if time.time() - t0 > timeout:
            raise TimeoutError("condition not reached")
        time.sleep(0.001)


SESS = [
    (160, 128, dict(amp=50.0)),
    (96, 80, dict(amp=120.0, color=True)),
    (137, 91, dict(amp=60.0, fps=60.0, f_high=8.0)),
    (200, 120, dict(amp=80.0, edge_aware=False)),
]


def test_served_sessions_equal_alone(oracle, torch_cuda):
    """Sessions open at different times and submit at different rates (some
    several frames at once); the dispatcher is held on alternate rounds so
    frames collect and ticks mix the sessions in changing combinations."""
    torch = torch_cuda
    F = 6
    data = [frames(w, h, F, seed=k + 41, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(SESS)]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    outs = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
            for (w, h, _) in SESS]
    torch.cuda.synchronize()
    srv = wc.Server(device=0, budget_bytes=8 << 30, max_streams=8)
    sids = [None] * len(SESS)
    nxt = [0] * len(SESS)
    step = 0
    while min(nxt) < F:
        srv.hold(step % 2 == 0)
        for k, (w, h, cfg) in enumerate(SESS):
            if sids[k] is None and step >= 2 * k:          # staggered arrivals
                sids[k] = srv.open(w, h, **cfg)
                wait_for(lambda: srv.poll(sids[k])["state"] == wc.SESSION_LIVE)
            if sids[k] is None or nxt[k] >= F:
                continue
            burst = 1 + (step + k) % 3                      # 1-3 frames at once
            for _ in range(burst):
                if nxt[k] < F and srv.submit(sids[k], d_in[k][nxt[k]], outs[k][nxt[k]]) == 0:
                    nxt[k] += 1
        step += 1
        time.sleep(0.002)
    srv.hold(False)
    srv.drain()
    st = srv.stats()
    assert st["frames"] == F * len(SESS)
    assert st["ticks"] < F * len(SESS)                      # frames shared ticks
    for k, (w, h, cfg) in enumerate(SESS):
        assert srv.poll(sids[k])["completed"] == F
        ref = alone(torch, w, h, cfg, data[k])
        want = oracle_u8(oracle, data[k], **cfg)
        for t in range(F):
            got = outs[k][t].cpu().numpy()
            assert np.array_equal(got, ref[t]), f"session {k} frame {t}"
            assert_close(got, want[t], cfg.get("color", False), f"session {k} frame {t}")
    srv.close()


def test_admission_against_budget(torch_cuda):
    torch = torch_cuda
    w, h = 160, 128
    cost = wc.lib().wema_cuda_batch_stream_bytes(wc.make_config(w, h))
    assert cost > 0
    srv = wc.Server(device=0, budget_bytes=2 * cost + cost // 2, max_streams=8)
    with pytest.raises(RuntimeError):
        srv.open(1920, 1080)                                # alone larger than the budget
    a = srv.open(w, h, amp=50.0)
    b = srv.open(w, h, amp=60.0)
    wait_for(lambda: srv.poll(b)["state"] == wc.SESSION_LIVE)
    c = srv.open(w, h, amp=70.0)                            # budget full: queued
    time.sleep(0.05)
    assert srv.poll(c)["state"] == wc.SESSION_QUEUED
    d_in = torch.from_numpy(frames(w, h, 3, seed=3)).cuda()
    o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
    assert srv.submit(c, d_in[0], o) == 1                   # refused while queued
    assert srv.poll(c)["dropped"] == 1
    outs_a = [torch.empty_like(o) for _ in range(3)]
    for t in range(3):
        assert srv.submit(a, d_in[t], outs_a[t]) == 0
    srv.close_session(a)                                    # pending frames still run
    wait_for(lambda: srv.poll(c)["state"] == wc.SESSION_LIVE)
    pa, pc = srv.poll(a), srv.poll(c)
    assert pa["state"] == wc.SESSION_CLOSED and pa["completed"] == 3
    assert pc["admission_wait_ms"] > 0
    st = srv.stats()
    assert st["sessions_live"] == 2 and st["sessions_queued"] == 0
    assert st["bytes_used"] == 2 * cost
    with pytest.raises(RuntimeError):
        srv.submit(a, d_in[0], o)                           # closed
    ref = alone(torch, w, h, dict(amp=50.0), frames(w, h, 3, seed=3))
    for t in range(3):
        assert np.array_equal(outs_a[t].cpu().numpy(), ref[t])
    srv.close()
