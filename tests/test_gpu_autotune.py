"""The autotuner: it picks one of the candidate positions-per-thread counts of
the temporal filter and reports the trial timings; the frames do not depend on
the choice (each position's arithmetic is the same), per stream and batched."""
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


def test_autotune_and_choice_independence(torch_cuda):
    torch = torch_cuda
    before = wc.iir_positions(0)
    u, report = wc.autotune(0)
    assert u in (2, 4, 8) and wc.iir_positions(0) == u and "->" in report
    w, h, F = 160, 96, 5
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 4, [1.2], [0.4], 14.0, 2.0)).frames(0, F)
    d = torch.from_numpy(u8).cuda()
    outs = {}
    for p in (2, 4, 8):
        wc.set_iir_positions(0, p)
        s = wc.Session(width=w, height=h, fps=30.0, amp=70.0)
        b = wc.Batch(device=0, max_streams=1)
        sid = b.add(w, h, fps=30.0, amp=70.0, state_fp64=True)
        got = []
        for t in range(F):
            o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
            ob = torch.empty_like(o)
            s.process_u8(d[t], o)
            b.tick([sid], [d[t]], [ob])
            b.sync()
            torch.cuda.synchronize()
            got.append((o.cpu().numpy(), ob.cpu().numpy()))
        outs[p] = got
        s.close()
        b.close()
    for p in (2, 8):
        for t in range(F):
            assert np.array_equal(outs[p][t][0], outs[4][t][0]), f"session, {p} positions, frame {t}"
            assert np.array_equal(outs[p][t][1], outs[4][t][1]), f"batched FP64 state, {p} positions, frame {t}"
    with pytest.raises(RuntimeError):
        wc.set_iir_positions(0, 3)
    wc.set_iir_positions(0, before)


def test_guided_rows_choice_independence(torch_cuda):
    """The guided filter's sweep gives the same frames for every segment
    height (its running sums restart at rows fixed in the frame), batched and
    per stream, on word-aligned and ragged frames."""
    torch = torch_cuda
    assert "guided sweep rows" in wc.autotune(0)[1]
    before = wc.guided_rows(0)
    F = 4
    cfgs = [(640, 480, dict(amp=90.0)), (137, 91, dict(amp=60.0)), (1920, 1080, dict(amp=40.0))]
    data = [torch.from_numpy(SynthVideo(SynthSpec(w, h, 30.0, 3 + k, [1.1], [0.4], 14.0, 2.0))
                             .frames(0, F)).cuda() for k, (w, h, _) in enumerate(cfgs)]
    outs = {}
    for rows in (16, 48, 128, 256):
        wc.set_guided_rows(0, rows)
        b = wc.Batch(device=0, max_streams=len(cfgs))
        ids = [b.add(w, h, **c) for (w, h, c) in cfgs]
        got = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
               for (w, h, _) in cfgs]
        for t in range(F):
            b.tick(ids, [d[t] for d in data], [g[t] for g in got])
        b.sync()
        outs[rows] = [[x.cpu().numpy() for x in g] for g in got]
        b.close()
    for rows in (16, 48, 256):
        for k in range(len(cfgs)):
            for t in range(F):
                assert np.array_equal(outs[rows][k][t], outs[128][k][t]), f"{rows} rows, stream {k}, frame {t}"
    # the per-stream path (shorter segments for latency) gives the batched frames
    for k, (w, h, c) in enumerate(cfgs):
        s = wc.Session(width=w, height=h, **c)
        for t in range(F):
            o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
            s.process_u8(data[k][t], o)
            s.sync()
            assert np.array_equal(o.cpu().numpy(), outs[128][k][t]), f"session, stream {k}, frame {t}"
        s.close()
    with pytest.raises(RuntimeError):
        wc.set_guided_rows(0, 40)
    wc.set_guided_rows(0, before)


def test_dwt_variants_choice_independence(torch_cuda):
    """Every tuning variant of the batched luma DWT kernels (CTAs per SM x
    lines per warp, forward and inverse) gives the same frames, bit for bit;
    the autotuner reports its trial and keeps a variant."""
    torch = torch_cuda
    report = wc.autotune(0)[1]
    assert "forward DWT level 0" in report and "inverse DWT level 0" in report
    keep = (wc.dwt_variant(0, False), wc.dwt_variant(0, True))
    F = 3
    cfgs = [(640, 480, dict(amp=90.0)), (137, 91, dict(amp=60.0)), (1920, 1080, dict(amp=40.0))]
    data = [torch.from_numpy(SynthVideo(SynthSpec(w, h, 30.0, 13 + k, [1.1], [0.4], 14.0, 2.0))
                             .frames(0, F)).cuda() for k, (w, h, _) in enumerate(cfgs)]
    outs = {}
    for v in range(9):
        wc.set_dwt_variant(0, False, v)
        wc.set_dwt_variant(0, True, (v + 4) % 9)
        b = wc.Batch(device=0, max_streams=len(cfgs))
        ids = [b.add(w, h, **c) for (w, h, c) in cfgs]
        got = [[torch.empty((h, w, 3), dtype=torch.uint8, device="cuda") for _ in range(F)]
               for (w, h, _) in cfgs]
        for t in range(F):
            b.tick(ids, [d[t] for d in data], [g[t] for g in got])
        b.sync()
        outs[v] = [[x.cpu().numpy() for x in g] for g in got]
        b.close()
    for v in range(1, 9):
        for k in range(len(cfgs)):
            for t in range(F):
                assert np.array_equal(outs[v][k][t], outs[0][k][t]), f"variant {v}, stream {k}, frame {t}"
    with pytest.raises(RuntimeError):
        wc.set_dwt_variant(0, False, 9)
    wc.set_dwt_variant(0, False, keep[0])
    wc.set_dwt_variant(0, True, keep[1])
