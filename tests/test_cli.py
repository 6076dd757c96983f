"""The reference CLI's command line over libwema_cuda (wema-cuda-cli): flag
checks and messages as main.c's parse_args (on the host), and on a GPU a raw
RGB24 file through it equal to the same stream through a session."""
import os
import subprocess

import numpy as np
import pytest

from wema_b200 import _build

CLI = _build.cli_path()


@pytest.fixture(scope="module", autouse=True)
def built():
    _build.build_cli()


def run(*args, **kw):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120, **kw)


def test_help():
    r = run("-h")
    assert r.returncode == 0 and "Usage:" in r.stderr and "--temporal-window" in r.stderr


@pytest.mark.parametrize("args,msg", [
    (["--bogus"], "Unknown option: --bogus"),
    (["--size", "64x48", "--fps", "30"], "Input file required (-i)"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "-a", "0"], "amplification factor must be positive"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--fl", "-1"], "low frequency must be non-negative"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--fh", "0"], "high frequency must be positive"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--fl", "3", "--fh", "2"],
     "Low frequency must be less than high frequency"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--temporal-window", "3"],
     "temporal window must be at least 4"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--temporal-window", "257"],
     "temporal window cannot exceed 256"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--batch", "0"], "batch size must be at least 1"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--batch", "257"], "batch size cannot exceed 256"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "--threads", "-1"], "thread count must be non-negative"),
    (["-i", "x.rgb", "--size", "64x48", "--fps", "30", "-a"], "-a requires an argument"),
    (["-i", "x.rgb", "--fps", "30"], "needs --size"),
    (["-i", "x.rgb", "--size", "64x", "--fps", "30"], "--size takes"),
])
def test_flag_errors(args, msg):
    r = run(*args)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_nyquist_clamp_rejects_empty_band(tmp_path):
    # --fl above the clamped --fh (fps/2 - 1e-4): rejected before any device work
    r = run("-i", str(tmp_path / "x.rgb"), "--size", "64x48", "--fps", "10", "--fl", "6")
    assert r.returncode == 1 and "Low frequency must be less than high frequency" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("extra,cfg", [
    ([], dict(threshold_form=1)),                                   # IIR luma: the batch route
    (["--batch", "1", "--no-edge-aware"], dict(edge_aware=False)),  # single-frame route, Gaussian
    (["--color"], dict(color=True)),
])
def test_cli_equals_session(oracle, tmp_path, extra, cfg):
    import torch
    from wema_b200 import cuda as wc
    from wema_b200.synth import SynthSpec, SynthVideo
    w, h, F = 96, 64, 5
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 9, [1.1], [0.4], 12.0, 2.0)).frames(0, F)
    src, dst = tmp_path / "in.rgb", tmp_path / "out.rgb"
    u8.tofile(src)
    r = run("-i", str(src), "-o", str(dst), "--size", f"{w}x{h}", "--fps", "30", "-a", "80",
            "--fl", "0.5", "--fh", "3", *extra)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(dst, np.uint8).reshape(F, h, w, 3)
    s = wc.Session(width=w, height=h, fps=30.0, amp=80.0, f_low=0.5, f_high=3.0, **cfg)
    d = torch.from_numpy(u8).cuda()
    for t in range(F):
        o = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        s.process_u8(d[t], o)
        torch.cuda.synchronize()
        assert np.array_equal(o.cpu().numpy(), got[t]), f"frame {t}"
    s.close()
    from oracle_frames import assert_close, oracle_u8
    want = oracle_u8(oracle, u8, fps=30.0, amp=80.0, f_low=0.5, f_high=3.0, **cfg)
    for t in range(F):
        assert_close(got[t], want[t], cfg.get("color", False), f"CLI frame {t}")


@pytest.mark.gpu
def test_cli_partial_frame_is_an_error(tmp_path):
    src = tmp_path / "in.rgb"
    np.zeros(64 * 48 * 3 + 10, np.uint8).tofile(src)
    r = run("-i", str(src), "-o", str(tmp_path / "o.rgb"), "--size", "64x48", "--fps", "30")
    assert r.returncode == 1 and "partial frame" in r.stderr
