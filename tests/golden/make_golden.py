"""Generates tests/golden/*.npz from the reference library itself.

Run where the reference was compiled (``make -C oracle ref``):

    python tests/golden/make_golden.py

Each fixture stores what the reference computed on seeded synthetic frames
(regenerated from the stored generator parameters; a SHA-256 of the input
bytes guards against generator drift):

* SHA-256 of the float32 stage buffers per frame (6-slot original
  coefficients, IIR deltas, amplified coefficients, reconstructed Y) - these
  stages are bit-exact in the oracle and on the GPU;
* the reference's u8 output frames (float output quantised the way the
  reference's writer does);
* the IIR design coefficients and warm-up counts for the benchmark bands;
* threshold probes: a frame's 6-slot coefficients with 64 entries replaced
  by consecutive floats around the threshold, and which of them the
  reference's coeff_amplify amplified - this pins the threshold to the bit.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

from oracle import Oracle, Reference  # noqa: E402
from wema_b200.synth import SynthSpec, SynthVideo  # noqa: E402

CASES = {
    "luma_iir_128": dict(size=(128, 128), frames=6, seed=21,
                         cfg=dict(fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, color=False,
                                  edge_aware=True)),
    "luma_iir_136x130": dict(size=(136, 130), frames=4, seed=22,
                             cfg=dict(fps=60.0, amp=120.0, f_low=0.5, f_high=3.0, color=False,
                                      edge_aware=True)),
    "color_iir_128": dict(size=(128, 128), frames=4, seed=23,
                          cfg=dict(fps=30.0, amp=120.0, f_low=0.5, f_high=3.0, color=True)),
    "batch_iir_128": dict(size=(128, 128), frames=6, seed=24, batch=True,
                          cfg=dict(fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, color=False,
                                   edge_aware=True)),
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def spec_for(case):
    w, h = case["size"]
    return SynthSpec(w, h, case["cfg"]["fps"], case["seed"], [1.2], [0.4], 20.0, 2.0)


def threshold_probe(O, orig, k=64):
    """Replaces k entries of orig by consecutive floats straddling the
    threshold (found as a fixed point, since the probes enter the sum)."""
    rng = np.random.default_rng(9)
    idx = np.sort(rng.choice(orig.size, k, replace=False)).astype(np.int64)
    orig = orig.copy()
    t = np.float32(O.threshold(orig))
    for _ in range(20):
        vals = np.array([t], np.float32).view(np.int32) + np.arange(-k // 2, k // 2, dtype=np.int32)
        orig[idx] = vals.view(np.float32) * np.where(np.arange(k) % 2 == 0, 1, -1).astype(np.float32)
        t_new = np.float32(O.threshold(orig))
        if t_new == t:
            break
        t = t_new
    return idx, orig


def main():
    O, R = Oracle(), Reference()
    meta = {}
    arrays = {}
    for name, case in CASES.items():
        w, h = case["size"]
        sv = SynthVideo(spec_for(case))
        u8 = sv.frames(0, case["frames"])
        rgb = O.u8_to_float(u8)
        cfg = dict(width=w, height=h, window=32, bilateral=False, use_iir=True, **case["cfg"])
        N, P = O.positions(w, h), w * h
        entry = {"input_sha": sha(u8), "spec": spec_for(case).__dict__, "cfg": cfg,
                 "frames": case["frames"], "stages": []}
        if case.get("batch"):
            s = R.stream(batch_size=case["frames"], **cfg)
            out = s.batch(rgb)
            arrays[name + "/out_u8"] = O.float_to_u8(out)
        else:
            s = R.stream(**cfg)
            outs = []
            for t in range(case["frames"]):
                o = s.process(rgb[t])
                outs.append(O.float_to_u8(o))
                st = {k: sha(s.get(i, N)) for k, i in (("orig6", 2), ("delta6", 3), ("amp6", 4))}
                st["gray_out"] = sha(s.get(1, P))
                if cfg["color"]:
                    st["out_f32"] = sha(o)
                entry["stages"].append(st)
            arrays[name + "/out_u8"] = np.stack(outs)
        meta[name] = entry
    bands = [(0.5, 3.0, 30.0), (0.5, 3.0, 60.0), (0.2, 0.6, 240.0), (0.5, 5.0, 30.0), (0.5, 14.9999, 30.0)]
    meta["iir_design"] = []
    for fl, fh, fs in bands:
        c, wu = R.iir_design(fl, fh, fs)
        meta["iir_design"].append({"band": [fl, fh, fs], "coef_hex": c.view(np.uint32).tolist(),
                                   "warmup": wu})
    meta["thrprobe"] = []
    for name in ("luma_iir_128", "color_iir_128"):
        case = CASES[name]
        w, h = case["size"]
        u8 = SynthVideo(spec_for(case)).frames(0, 1)
        y = O.gray(O.u8_to_float(u8)[0])
        orig, _ = O.dwt_forward(y)
        probes, orig = threshold_probe(O, orig)
        delta = np.zeros_like(orig)
        delta[probes] = 1.0
        out = R.coeff_amplify(delta, orig, 1.0, w, h)
        mask = (out[probes] != orig[probes]).astype(np.uint8)
        arrays[f"thrprobe/{name}/orig"] = orig
        arrays[f"thrprobe/{name}/idx"] = probes
        arrays[f"thrprobe/{name}/mask"] = mask
        meta["thrprobe"].append({"case": name, "size": [w, h], "amplified": int(mask.sum())})
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.npz"))


if __name__ == "__main__":
    main()
