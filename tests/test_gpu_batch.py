"""Batched streams (wema_cuda_batch_*): every stream's frames in a mixed batch
are bit-identical to the same stream run alone through a wema_cuda_session,
whatever the mix (sizes, luma / colour, edge-aware / Gaussian, streams that
skip ticks, streams added and removed between ticks); one batched stream is
also checked against the oracle (u8 within 1 LSB, colour bit-exact)."""
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


# (width, height, config): uneven sizes, odd level inputs, both modes
STREAMS = [
    (160, 128, dict(amp=50.0)),
    (200, 120, dict(amp=80.0, edge_aware=False)),
    (96, 80, dict(amp=120.0, color=True)),
    (320, 240, dict(amp=30.0, f_high=5.0)),
    (137, 91, dict(amp=60.0, color=True, fps=60.0, f_high=8.0)),
    (64, 48, dict(amp=40.0)),
]


def alone(torch, w, h, cfg, u8):
    """The stream's outputs through a plain session, one frame at a time."""
    s = wc.Session(width=w, height=h, **cfg)
    d_in = torch.from_numpy(u8).cuda()
    outs = []
    for t in range(u8.shape[0]):
        o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        s.process_u8(d_in[t], o)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
    thr = s.read(wc.READ_THRESHOLD)[0]
    s.close()
    return outs, thr


def test_batch_matches_streams_alone(torch_cuda):
    torch = torch_cuda
    F = 6
    data = [frames(w, h, F, seed=k + 1, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(STREAMS)]
    b = wc.Batch(device=0, max_streams=16)
    ids = [b.add(w, h, **cfg) for (w, h, cfg) in STREAMS]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    outs = [[None] * F for _ in STREAMS]
    # stream k takes part in tick t when (t + k) % 3 != 2, so streams skip ticks
    # and every tick mixes a different subset; each stream still sees its frames
    # in order
    nxt = [0] * len(STREAMS)
    tick = 0
    while min(nxt) < F:
        sel = [k for k in range(len(STREAMS)) if nxt[k] < F and ((tick + k) % 3 != 2 or tick > 3 * F)]
        tick += 1
        if not sel:
            continue
        o_t = [torch.empty((STREAMS[k][1], STREAMS[k][0], 3), dtype=torch.uint8, device="cuda") for k in sel]
        b.tick([ids[k] for k in sel], [d_in[k][nxt[k]] for k in sel], o_t)
        b.sync()
        for k, o in zip(sel, o_t):
            outs[k][nxt[k]] = o.cpu().numpy()
            nxt[k] += 1
    st = b.stats()
    assert st["live"] == len(STREAMS)
    for k, (w, h, cfg) in enumerate(STREAMS):
        ref, thr = alone(torch, w, h, cfg, data[k])
        for t in range(F):
            assert np.array_equal(outs[k][t], ref[t]), f"stream {k} frame {t}"
        assert b.threshold(ids[k]) == thr, f"stream {k} threshold"
    b.close()


def test_batch_back_to_back_ticks(torch_cuda):
    """Ticks issued without waiting (consecutive ticks overlap on the device)
    give the same frames as streams run alone."""
    torch = torch_cuda
    F = 5
    data = [frames(w, h, F, seed=k + 31, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(STREAMS)]
    b = wc.Batch(device=0, max_streams=len(STREAMS))
    ids = [b.add(w, h, **cfg) for (w, h, cfg) in STREAMS]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    outs = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
            for (w, h, _) in STREAMS]
    torch.cuda.synchronize()
    for t in range(F):
        b.tick(ids, [d[t] for d in d_in], [o[t] for o in outs])
    b.sync()
    for k, (w, h, cfg) in enumerate(STREAMS):
        ref, _ = alone(torch, w, h, cfg, data[k])
        for t in range(F):
            assert np.array_equal(outs[k][t].cpu().numpy(), ref[t]), f"stream {k} frame {t}"
    b.close()


def test_batch_add_remove(torch_cuda):
    torch = torch_cuda
    F = 4
    (w0, h0, c0), (w1, h1, c1) = STREAMS[0], STREAMS[2]
    u0, u1 = frames(w0, h0, 2 * F, seed=11), frames(w1, h1, F, seed=12)
    b = wc.Batch(device=0, max_streams=2)
    a = b.add(w0, h0, **c0)
    d0, d1 = torch.from_numpy(u0).cuda(), torch.from_numpy(u1).cuda()
    got0 = []
    for t in range(F):
        o = torch.empty((h0, w0, 3), dtype=torch.uint8, device="cuda")
        b.tick([a], [d0[t]], [o])
        b.sync()
        got0.append(o.cpu().numpy())
    c = b.add(w1, h1, **c1)
    with pytest.raises(RuntimeError):
        b.add(w1, h1, **c1)                  # over max_streams
    got1 = []
    for t in range(F):
        o0 = torch.empty((h0, w0, 3), dtype=torch.uint8, device="cuda")
        o1 = torch.empty((h1, w1, 3), dtype=torch.uint8, device="cuda")
        b.tick([c, a], [d1[t], d0[F + t]], [o1, o0])
        b.sync()
        got0.append(o0.cpu().numpy())
        got1.append(o1.cpu().numpy())
    b.remove(a)
    with pytest.raises(RuntimeError):
        b.tick([a], [d0[0]], [o0])           # removed
    ref0, _ = alone(torch, w0, h0, c0, u0)
    ref1, _ = alone(torch, w1, h1, c1, u1)
    for t in range(2 * F):
        assert np.array_equal(got0[t], ref0[t]), f"stream a frame {t}"
    for t in range(F):
        assert np.array_equal(got1[t], ref1[t]), f"stream c frame {t}"
    b.close()


@pytest.mark.parametrize("color", [False, True])
def test_batch_against_oracle(oracle, torch_cuda, color):
    torch = torch_cuda
    w, h, F = 160, 128, 4
    u8 = frames(w, h, F, seed=21)
    rgb = oracle.u8_to_float(u8)
    so = oracle.stream(width=w, height=h, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, window=32,
                       edge_aware=True, bilateral=False, color=color, use_iir=True)
    b = wc.Batch(device=0, max_streams=2)
    other = b.add(200, 120, amp=80.0)        # a neighbour in every tick
    sid = b.add(w, h, amp=50.0, f_low=0.5, f_high=3.0, color=color)
    d = torch.from_numpy(u8).cuda()
    dn = torch.from_numpy(frames(200, 120, F, seed=22)).cuda()
    for t in range(F):
        o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        on = torch.empty((120, 200, 3), dtype=torch.uint8, device="cuda")
        b.tick([other, sid], [dn[t], d[t]], [on, o])
        b.sync()
        ref = oracle.float_to_u8(so.process(rgb[t]))
        diff = np.abs(ref.astype(int) - o.cpu().numpy().astype(int))
        if color:
            assert diff.max() == 0, f"frame {t}: colour output"
        else:
            assert diff.max() <= 1, f"frame {t}: {diff.max()} LSB"
    b.close()


def test_batch_stage_timing(torch_cuda):
    """Per-stage device times of batched ticks: every stage the tick ran is
    timed, and timing does not change the frames."""
    torch = torch_cuda
    (w, h, cfg) = STREAMS[0]
    u8 = frames(w, h, 4, seed=51)
    d = torch.from_numpy(u8).cuda()
    outs = {}
    for timed in (False, True):
        b = wc.Batch(device=0, max_streams=1)
        sid = b.add(w, h, **cfg)
        b.set_timing(timed)
        o = [torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(4)]
        for t in range(4):
            b.tick([sid], [d[t]], [o[t]])
        times, n = b.stage_times()
        if timed:
            assert n == 4
            for k in ("fwd_dwt_level0", "fwd_dwt_levels", "threshold", "temporal_amplify",
                      "inv_dwt_levels", "inv_dwt_level0", "luma_transfer"):
                assert times[k] > 0, k
        else:
            assert n == 0
        outs[timed] = [x.cpu().numpy() for x in o]
        b.close()
    for t in range(4):
        assert np.array_equal(outs[False][t], outs[True][t])


def test_batch_tick_host_equals_device(oracle, torch_cuda):
    """Host-frame ticks (pinned and pageable buffers, double-buffered staging)
    give the device ticks' frames, and the oracle's."""
    torch = torch_cuda
    F = 5
    sel = [STREAMS[0], STREAMS[2], STREAMS[4]]
    data = [frames(w, h, F, seed=k + 61, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(sel)]
    dev = wc.Batch(device=0, max_streams=4)
    hst = wc.Batch(device=0, max_streams=4)
    ids_d = [dev.add(w, h, **cfg) for (w, h, cfg) in sel]
    ids_h = [hst.add(w, h, **cfg) for (w, h, cfg) in sel]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    ref = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)] for (w, h, _) in sel]
    # stream 0 pinned tensors, the others pageable numpy arrays
    h_in = [[torch.from_numpy(data[0][t]).pin_memory() for t in range(F)]] + \
           [[np.ascontiguousarray(data[k][t]) for t in range(F)] for k in (1, 2)]
    h_out = [[torch.empty((sel[0][1], sel[0][0], 3), dtype=torch.uint8).pin_memory() for _ in range(F)]] + \
            [[np.empty((h, w, 3), np.uint8) for _ in range(F)] for (w, h, _) in sel[1:]]
    for t in range(F):
        dev.tick(ids_d, [d[t] for d in d_in], [r[t] for r in ref])
        hst.tick_host(ids_h, [x[t] for x in h_in], [x[t] for x in h_out])
    dev.sync()
    hst.sync()
    for k, (w, h, cfg) in enumerate(sel):
        want = oracle_u8(oracle, data[k], **cfg)
        for t in range(F):
            got = h_out[k][t].numpy() if hasattr(h_out[k][t], "numpy") else h_out[k][t]
            assert np.array_equal(got, ref[k][t].cpu().numpy()), f"stream {k} frame {t}"
            assert_close(got, want[t], cfg.get("color", False), f"stream {k} frame {t}")
    dev.close()
    hst.close()


@pytest.mark.parametrize("overlap", [True, False])
def test_batch_tick_host_contiguous_frames(torch_cuda, overlap):
    """Host frames back to back in one pinned arena (the copies coalesce into
    one per direction, across sizes whose frames are 256-byte multiples and
    not) give the device ticks' frames, with and without the copies in
    overlapping the previous tick."""
    torch = torch_cuda
    F = 5
    sel = [(160, 128, dict(amp=50.0)), (320, 240, dict(amp=30.0, f_high=5.0)),
           (137, 91, dict(amp=60.0, fps=60.0, f_high=8.0)), (96, 80, dict(amp=120.0, color=True))]
    data = [frames(w, h, F, seed=k + 81, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(sel)]
    fb = [3 * w * h for (w, h, _) in sel]
    offs = np.concatenate([[0], np.cumsum(fb)])
    arena_in = [torch.empty(int(offs[-1]), dtype=torch.uint8).pin_memory() for _ in range(F)]
    arena_out = [torch.empty(int(offs[-1]), dtype=torch.uint8).pin_memory() for _ in range(F)]
    for t in range(F):
        for k in range(len(sel)):
            arena_in[t][offs[k]:offs[k + 1]].copy_(torch.from_numpy(data[k][t].reshape(-1)))
    dev = wc.Batch(device=0, max_streams=4)
    hst = wc.Batch(device=0, max_streams=4)
    hst.set_host_overlap(overlap)
    ids_d = [dev.add(w, h, **cfg) for (w, h, cfg) in sel]
    ids_h = [hst.add(w, h, **cfg) for (w, h, cfg) in sel]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    ref = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)] for (w, h, _) in sel]
    for t in range(F):
        dev.tick(ids_d, [d[t] for d in d_in], [r[t] for r in ref])
        hst.tick_host(ids_h, [arena_in[t][offs[k]:offs[k + 1]] for k in range(len(sel))],
                      [arena_out[t][offs[k]:offs[k + 1]] for k in range(len(sel))])
    dev.sync()
    hst.sync()
    for k, (w, h, _) in enumerate(sel):
        for t in range(F):
            got = arena_out[t][offs[k]:offs[k + 1]].numpy().reshape(h, w, 3)
            assert np.array_equal(got, ref[k][t].cpu().numpy()), f"stream {k} frame {t}"
    dev.close()
    hst.close()


def test_batch_graph_replay_equals_launches(oracle, torch_cuda):
    """Steady ticks replayed as CUDA graphs - with the streams in 1, 2 or 4
    pipelined groups - give the frames of the same ticks launched kernel by
    kernel, through changes of the tick's stream set (a stream skipping ticks,
    one added, one removed: each change captures again), ticks issued back to
    back (synchronised every third tick only), and the oracle's."""
    torch = torch_cuda
    F = 7
    sel = [STREAMS[0], STREAMS[2], STREAMS[3], STREAMS[4]]
    data = [frames(w, h, F, seed=k + 91, fps=cfg.get("fps", 30.0)) for k, (w, h, cfg) in enumerate(sel)]
    d_in = [torch.from_numpy(u).cuda() for u in data]
    modes = [(False, 1), (True, 1), (True, 2), (True, 4)]
    outs = {}
    for graphs, groups in modes:
        b = wc.Batch(device=0, max_streams=8)
        b.set_graphs(graphs)
        b.set_groups(groups)
        ids = [b.add(w, h, **cfg) for (w, h, cfg) in sel[:3]]
        got = [[None] * F for _ in sel]
        nxt = [0] * len(sel)
        for tick in range(F + 4):
            if tick == 3:
                b.sync()
                ids.append(b.add(sel[3][0], sel[3][1], **sel[3][2]))   # joins late
            live = [k for k in range(len(ids)) if nxt[k] < F and not (k == 1 and tick in (4, 5))]
            if tick == 8 and 0 in live:
                live.remove(0)
            if not live:
                continue
            o = [torch.empty((sel[k][1], sel[k][0], 3), dtype=torch.uint8, device="cuda") for k in live]
            b.tick([ids[k] for k in live], [d_in[k][nxt[k]] for k in live], o)
            if tick % 3 == 2:
                b.sync()
            for k, x in zip(live, o):
                got[k][nxt[k]] = x     # read after the last tick
                nxt[k] += 1
        b.sync()
        outs[(graphs, groups)] = [[None if x is None else x.cpu().numpy() for x in row] for row in got]
        b.close()
    base = outs[modes[0]]
    for k, (w, h, cfg) in enumerate(sel):
        want = oracle_u8(oracle, data[k], **cfg)
        for t in range(F):
            for m in modes[1:]:
                if base[k][t] is None:
                    assert outs[m][k][t] is None
                    continue
                assert np.array_equal(outs[m][k][t], base[k][t]), f"mode {m} stream {k} frame {t}"
            if base[k][t] is not None:
                assert_close(base[k][t], want[t], cfg.get("color", False), f"stream {k} frame {t}")
