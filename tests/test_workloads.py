"""The benchmark workloads' generators: the mixed 48-stream set and the
served Poisson session list have the shapes and distributions they state."""
import numpy as np

from wema_b200 import synth as S


def test_mixed_streams():
    mix = S.mixed_streams(seed=7)
    sizes = [(s.width, s.height, c["fps"]) for s, c in mix]
    assert sizes.count((640, 480, 30.0)) == 16 and sizes.count((1280, 720, 30.0)) == 16
    assert sizes.count((1920, 1080, 60.0)) == 12 and sizes.count((3840, 2160, 30.0)) == 4
    assert len({s.seed for s, _ in mix}) == 48                    # every stream its own seed
    for s, c in mix:
        assert 1 <= len(s.disc_freq) <= 3 and all(0.5 <= f <= 4.0 for f in s.disc_freq)
        assert 20.0 <= c["amp"] <= 150.0 and 16 <= c["window"] <= 64
        assert (c["f_low"], c["f_high"]) == (0.5, 5.0) and c["edge_aware"] and not c["color"]
    assert S.mixed_streams(seed=7)[5][1] == mix[5][1]            # seeded


def test_served_sessions_statistics():
    H = 2000.0
    ss = S.served_sessions(seed=3, horizon_s=H)
    opens = np.array([t0 for t0, _, _, _ in ss if t0 > 0])
    rate = len(opens) / H
    assert abs(rate - 2.0) < 0.15                                # Poisson, mean 2 / s
    gaps = np.diff(np.sort(opens))
    assert abs(gaps.mean() - 0.5) < 0.05 and abs(gaps.std() / gaps.mean() - 1.0) < 0.1   # exponential
    lengths = np.array([t1 - t0 for t0, t1, _, _ in ss if t0 > 0 and t1 < H])
    assert lengths.min() >= 5.0 - 1e-9 and lengths.max() <= 60.0 + 1e-9
    lg = np.log(lengths)
    assert abs(lg.mean() - (np.log(5) + np.log(60)) / 2) < 0.1  # log-uniform
    res = [s.width for _, _, s, _ in ss]
    frac = {w: res.count(w) / len(res) for w in (640, 1280, 1920, 3840)}
    for w, p in ((640, 0.40), (1280, 0.30), (1920, 0.25), (3840, 0.05)):
        assert abs(frac[w] - p) < 0.04, (w, frac[w])
    fps = [c["fps"] for _, _, _, c in ss]
    assert set(fps) == {30.0, 60.0} and abs(fps.count(60.0) / len(fps) - 0.5) < 0.05
    alive0 = [x for x in ss if x[0] == 0.0]
    assert 20 <= len(alive0) <= 70                               # steady state: about 2 x 22 s
