"""The oracle's u8 output frames for a stream, for tests that compare a
runtime form (host ticks, the CLI, the served loop, restored snapshots) with
the oracle directly as well as with a plain session."""
import numpy as np

ORACLE_KEYS = ("amp", "f_low", "f_high", "window", "edge_aware", "bilateral", "color", "use_iir")


def oracle_cfg(fps=30.0, **kw):
    """A stream's settings as the library's config defaults fill them in
    (wema_cuda_config_default: amp 120, 0.5 Hz, f_high = fps/2 - 1e-4 in
    FP32, window 32, edge-aware, IIR, luma)."""
    f32 = np.float32
    cfg = dict(fps=fps, amp=120.0, f_low=0.5,
               f_high=float(f32(f32(fps) / f32(2.0) - f32(0.0001))), window=32,
               edge_aware=True, bilateral=False, color=False, use_iir=True)
    cfg.update({k: v for k, v in kw.items() if k in ORACLE_KEYS})
    return cfg


def oracle_u8(oracle, u8, fps=30.0, threshold_form=0, **kw):
    """u8: [F][h][w][3] RGB24 frames; kw: the stream's Session/Batch settings.
    Returns the oracle's RGB24 output per frame, through the single-frame
    route (wema_process_frame), or the batch route (wema_batch_process) for
    the batch threshold form."""
    F, h, w = u8.shape[:3]
    rgb = oracle.u8_to_float(u8)
    so = oracle.stream(width=w, height=h, **oracle_cfg(fps, **kw))
    if threshold_form == 1:
        out = oracle.float_to_u8(so.batch(rgb))
    else:
        out = np.stack([oracle.float_to_u8(so.process(rgb[t])) for t in range(F)])
    so.close()
    return out


def assert_close(got, ref, color, what=""):
    """Colour output bit-exact, luma output within 1 LSB."""
    d = np.abs(np.asarray(got).astype(np.int16) - np.asarray(ref).astype(np.int16))
    bar = 0 if color else 1
    assert d.max() <= bar, f"{what}: {d.max()} LSB from the oracle"
