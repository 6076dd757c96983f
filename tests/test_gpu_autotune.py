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
