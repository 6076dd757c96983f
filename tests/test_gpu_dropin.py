"""The reference API, called from C11 (tests/c/dropin.c compiled against
include/ and linked with libwema_cuda), against the oracle.

The C program makes the same calls as the reference CLI (main.c:278-488):
wema_init, the flag fields, wema_init_color / wema_init_iir[_color], then
wema_batch_process or wema_process_frame; plus the stage APIs (dwt_*,
iir_temporal_*, coeff_amplify, temporal_buffer_* / temporal_filter_apply).
"""
import os
import subprocess

import numpy as np
import pytest

from wema_b200 import _build
from wema_b200.synth import SynthSpec, SynthVideo

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    lib = _build.cuda_lib_path()
    exe = str(tmp_path_factory.mktemp("c") / "dropin")
    subprocess.run(["gcc", "-std=c11", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "dropin.c"), "-L", os.path.dirname(lib),
                    "-lwema_cuda", "-Wl,-rpath," + os.path.dirname(lib), "-o", exe], check=True)
    return exe


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    return r.stdout


def u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("color,batch,edge,use_iir,bil", [
    (False, 1, True, True, False),     # wema_process_frame, IIR luma, guided filter
    (True, 1, True, True, False),      # IIR colour
    (False, 4, True, True, False),     # the default CLI route: wema_batch_process
    (False, 1, False, True, False),    # Gaussian fallback
    (False, 1, True, False, True),     # window mode with bilateral
])
def test_pipeline_from_c(oracle, dropin, tmp_path, color, batch, edge, use_iir, bil):
    w, h, F, ws = 160, 128, 10, 6
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 31, [1.4], [0.5], 20.0, 2.0)).frames(0, F)
    rgb = oracle.u8_to_float(u8)
    fin, fout = tmp_path / "in.f32", tmp_path / "out.f32"
    rgb.tofile(fin)
    out = run(dropin, "pipeline", w, h, 30.0, 80.0, 0.5, 3.0, ws, int(edge), int(bil), int(color),
              int(use_iir), batch, F, fin, fout)
    got = np.fromfile(fout, np.float32).reshape(F, h, w, 3)
    so = oracle.stream(width=w, height=h, fps=30.0, amp=80.0, f_low=0.5, f_high=3.0, window=ws,
                       edge_aware=edge, bilateral=bil, color=color, use_iir=use_iir)
    ref = so.batch(rgb) if batch > 1 else np.stack([so.process(rgb[t]) for t in range(F)])
    if color:
        assert np.array_equal(u32(got), u32(ref))
    d = np.abs(oracle.float_to_u8(got).astype(int) - oracle.float_to_u8(ref).astype(int))
    assert d.max() <= 1
    if use_iir:
        assert f"frames_processed {so.lib.orc_stream_frames_processed(so.h)}" in out


@pytest.mark.parametrize("w,h", [(160, 128), (136, 130), (37, 29)])
def test_dwt_from_c(oracle, dropin, tmp_path, w, h):
    rng = np.random.default_rng(w)
    img = rng.random((h, w), dtype=np.float32)
    img.tofile(tmp_path / "img")
    run(dropin, "dwt", w, h, tmp_path / "img", tmp_path / "flat", tmp_path / "low", tmp_path / "inv")
    flat_o, low_o = oracle.dwt_forward(img)
    assert np.array_equal(u32(np.fromfile(tmp_path / "flat", np.float32)), u32(flat_o))
    assert np.array_equal(u32(np.fromfile(tmp_path / "low", np.float32)), u32(low_o))
    inv_o = oracle.dwt_inverse(flat_o, low_o, w, h)
    assert np.array_equal(u32(np.fromfile(tmp_path / "inv", np.float32)), u32(inv_o.ravel()))


def test_iir_from_c(oracle, dropin, tmp_path):
    n, F = 1003, 12
    x = np.random.default_rng(4).standard_normal((F, n)).astype(np.float32)
    x.tofile(tmp_path / "x")
    out = run(dropin, "iir", n, F, 0.5, 3.0, 30.0, tmp_path / "x", tmp_path / "y")
    y = np.fromfile(tmp_path / "y", np.float32).reshape(F, n)
    assert np.array_equal(u32(y), u32(oracle.iir_run(x, 0.5, 3.0, 30.0)))
    c, wu = oracle.iir_design(0.5, 3.0, 30.0)
    assert f"frames_processed {wu + F} warmup {wu}" in out


def test_coeff_amplify_from_c(oracle, dropin, tmp_path):
    w, h = 160, 128
    u8 = SynthVideo(SynthSpec(w, h, 30.0, 5, [1.0], [0.4], 20.0, 2.0)).frame(0)
    orig, _ = oracle.dwt_forward(oracle.gray(oracle.u8_to_float(u8)))
    delta = (np.random.default_rng(1).standard_normal(orig.size) * 0.01).astype(np.float32)
    orig.tofile(tmp_path / "o")
    delta.tofile(tmp_path / "d")
    run(dropin, "amp", w, h, 50.0, tmp_path / "o", tmp_path / "d", tmp_path / "a")
    ref = oracle.amplify(delta, orig, 50.0, oracle.threshold(orig), w, h)
    assert np.array_equal(u32(np.fromfile(tmp_path / "a", np.float32)), u32(ref))


@pytest.mark.parametrize("bil", [0, 1])
def test_window_from_c(oracle, dropin, tmp_path, bil):
    w, h, ws, F = 64, 48, 8, 11
    N = oracle.positions(w, h)
    frames = np.random.default_rng(7).standard_normal((F, N)).astype(np.float32) * 0.05
    frames.tofile(tmp_path / "f")
    out = run(dropin, "window", w, h, ws, bil, F, tmp_path / "f", tmp_path / "d")
    got = np.fromfile(tmp_path / "d", np.float32)
    head = F % ws
    ring = np.empty((N, ws), np.float32)
    for t in range(F):
        ring[:, t % ws] = frames[t]
    ref = oracle.window_apply(ring, ws, head, bil)
    rel = np.linalg.norm(got.astype(np.float64) - ref) / np.linalg.norm(ref.astype(np.float64))
    assert rel <= 1e-5
    assert f"output_count {ws - ws // 2} head {head}" in out
