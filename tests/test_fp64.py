"""Pins the FP64 re-evaluation (oracle/fp64.py) against the bit-exact FP32
restatement: the two must differ only by FP32 rounding, so that the FP64
module can serve as the error reference for every FP32 result."""
import numpy as np
import pytest

import fp64
from wema_b200.synth import SynthSpec, SynthVideo


def unique_slots(flat6, dims):
    """The three unique slots of each level of a 6-slot array, concatenated
    in the FP64 module's order (level, slot, row, column)."""
    out, k6 = [], 0
    for (sw, sh) in dims:
        n = sw * sh
        out.append(flat6[k6: k6 + 3 * n])
        k6 += 6 * n
    return np.concatenate(out)


@pytest.mark.parametrize("w,h", [(64, 48), (37, 29), (160, 120), (33, 17), (96, 80)])
def test_dwt_fp64_against_fp32(oracle, w, h):
    rng = np.random.default_rng(w * 1000 + h)
    img = rng.random((h, w))
    bands, low = fp64.dwt_forward(img)
    rec = fp64.dwt_inverse(bands, low, w, h)
    assert np.abs(rec - img).max() < 1e-12                 # perfect reconstruction
    flat6, lp = oracle.dwt_forward(img.astype(np.float32))
    flat = np.concatenate([b.ravel() for lvl in bands for b in lvl])
    ref = unique_slots(flat6, oracle.subband_dims(w, h)).astype(np.float64)
    assert np.abs(flat - ref).max() < 2e-6                  # FP32 rounding of values <= ~3
    assert np.abs(low.ravel() - lp.astype(np.float64)).max() < 2e-6


@pytest.mark.parametrize("band", [(0.5, 3.0, 30.0), (0.5, 5.0, 60.0), (0.2, 0.6, 240.0)])
def test_iir_design_fp64_against_fp32(oracle, band):
    c32, wu32 = oracle.iir_design(*band)
    c64, wu64 = fp64.iir_design(*band)
    assert wu32 == wu64
    assert np.max(np.abs(c32.astype(np.float64) - c64) / np.abs(c64)) < 1e-6


def test_stream_fp64_against_fp32(oracle):
    w, h, F = 96, 80, 5
    spec = SynthSpec(w, h, 30.0, 3, [1.1], [0.4], 16.0, 2.0)
    u8 = SynthVideo(spec).frames(0, F)
    s32 = oracle.stream(width=w, height=h, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0)
    c32, _ = oracle.iir_design(0.5, 3.0, 30.0)
    s64 = fp64.Stream64(w, h, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, coef=c32)
    dims = oracle.subband_dims(w, h)
    rgb = oracle.u8_to_float(u8)
    for t in range(F):
        out32 = s32.process(rgb[t])
        orig6 = s32.get(2, 10 ** 6)
        thr = oracle.threshold(orig6)
        out64 = s64.process(u8[t], thr=thr)                 # same mask as the FP32 path
        d32 = unique_slots(s32.get(3, 10 ** 6), dims).astype(np.float64)
        d64 = s64.last["delta"]
        # the band-passed delta is a small difference of large terms (right
        # after the preseed it is ~1e-3 of the coefficients), so FP32 rounding
        # shows relative to the coefficients (amplified by the recursion), not
        # to the delta itself
        assert np.linalg.norm(d32 - d64) <= 1e-5 * np.linalg.norm(s64.last["coef"]), f"frame {t} delta"
        assert np.abs(out32.astype(np.float64) - out64).max() * 255.0 < 0.05, f"frame {t} output"


@pytest.mark.parametrize("w,h", [(64, 48), (37, 29), (9, 9)])
def test_box_and_guided_fp64_against_fp32(oracle, w, h):
    """The clipped-window box mean and the guided filter (r 4, eps 0.01) agree
    with the FP32 restatement to FP32 rounding (its running prefix sums lose a
    few ulp of the row total)."""
    rng = np.random.default_rng(w * h)
    I = rng.random((h, w))
    p = 0.05 * rng.standard_normal((h, w))
    b64 = fp64.box(I)
    b32 = oracle.box(I.astype(np.float32)).astype(np.float64)
    assert np.abs(b64 - b32).max() < 1e-5
    q64 = fp64.guided(I, p)
    q32 = oracle.guided(I.astype(np.float32), p.astype(np.float32)).astype(np.float64)
    assert np.abs(q64 - q32).max() < 1e-4
