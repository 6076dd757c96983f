"""FP64 re-evaluation of the per-frame path (test infrastructure only).

The reference computes in FP32 (and the C restatement in oracle/wema_oracle.c
reproduces its rounding bit for bit); this module evaluates the same steps in
double precision from the mathematical definitions, so every FP32 result can
state its error against it.  Steps and the reference lines they follow:

* u8 -> [0,1] and Y = .299 R + .587 G + .114 B      wema.c:42-51, ffmpeg_io.c:293
* level count and subband sizes                      dwt.c:588-621
* CDF 9/7 lifting, rows then columns, whole-sample
  symmetric extension, K scaling                     dwt.c:31-107, 369-473
* inverse: columns then rows, steps reversed         dwt.c:109-170, 475-582
* Butterworth HP(f_low) + LP(f_high) biquads in
  DF-II transposed form, preseed of `warmup` steps
  on the first frame, warmup = max(30, 7 fs/(2 pi fl)) iir_filter.c:36-154, 181-264, 376-471
* threshold = 0.2 x mean |coefficient| over the
  detail positions (the reference's 6-slot array
  holds every unique position twice)                 wema.c:719-723
* out = orig + [|orig| > thr] alpha_l delta,
  alpha_0 = alpha / 2, 15-frame quadratic fade-in    wema.c:714-744, 831-839
* guided filter r = 4, eps = 0.01, box means with
  the window clipped at the borders (rows, then
  columns), guide = input Y, p = output Y - input Y  wema.c:114-230
* RGB out = clamp01(RGB + q), u8 = floor(255 v + 0.5) wema.c:289-335, ffmpeg_io.c:305-310

Options isolate one precision effect at a time: `coef` takes the FP32-designed
biquad coefficients (promoted) instead of the FP64 design, and a caller may
pass the threshold to use (so a comparison is not dominated by coefficients
that sit on the threshold and flip the mask).

Frames whose level inputs are all of even size are represented exactly
(every config resolution except 1920x1080, whose level-4 input is 240x135);
for odd sizes the missing odd-index subband entries are taken as zero here,
whereas the reference keeps the previous level's values there, so compare
such frames on the output only.
"""
from __future__ import annotations

import math

import numpy as np

ALPHA, BETA, GAMMA, DELTA = -1.586134342059924, -0.052980118572961, 0.882911075530934, 0.443506852043971
K = 1.149604398860241


def levels(w: int, h: int) -> int:
    m, l = min(w, h), 0
    while m >= 16 and l < 4:
        m //= 2
        l += 1
    return max(l, 1)


def gray(rgb: np.ndarray) -> np.ndarray:
    """rgb: [..., 3] in [0,1] (float64)."""
    return 0.299 * rgb[..., 0] + 0.587 * rgb[..., 1] + 0.114 * rgb[..., 2]


# ------------------------------------------------------------------ lifting
def _predict(e, o, n, c):
    """o[i] += c (e[i] + e[i+1]); the right neighbour mirrors at the end."""
    ne, no = e.shape[-1], o.shape[-1]
    er = np.empty_like(o)
    if ne > no:                           # n odd: every odd sample has a right even
        er[...] = e[..., 1: no + 1]
    else:                                 # n even: the last one mirrors
        er[..., : no - 1] = e[..., 1: no]
        er[..., no - 1] = e[..., no - 1]
    o += c * (e[..., :no] + er)


def _update(e, o, n, c):
    """e[i] += c (o[i-1] + o[i]); both ends mirror."""
    ne, no = e.shape[-1], o.shape[-1]
    ol = np.empty_like(e)
    orr = np.empty_like(e)
    ol[..., 0] = o[..., 0]
    ol[..., 1:] = o[..., : ne - 1]
    orr[..., :no] = o
    if ne > no:                           # n odd: the last even sample has no right odd
        orr[..., no] = o[..., no - 1]
    e += c * (ol + orr)


def lift_fwd(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Forward 9/7 along the last axis: (low, high)."""
    n = x.shape[-1]
    e = x[..., 0::2].copy()
    o = x[..., 1::2].copy()
    if n < 2:
        return e, o
    _predict(e, o, n, ALPHA)
    _update(e, o, n, BETA)
    _predict(e, o, n, GAMMA)
    _update(e, o, n, DELTA)
    return e / K, o * K


def lift_inv(e: np.ndarray, o: np.ndarray) -> np.ndarray:
    n = e.shape[-1] + o.shape[-1]
    e = e * K
    o = o / K
    if n >= 2:
        _update(e, o, n, -DELTA)
        _predict(e, o, n, -GAMMA)
        _update(e, o, n, -BETA)
        _predict(e, o, n, -ALPHA)
    x = np.empty(e.shape[:-1] + (n,), dtype=e.dtype)
    x[..., 0::2] = e
    x[..., 1::2] = o
    return x


def dwt_forward(img: np.ndarray):
    """-> (bands, lowpass): bands[l] = (LH, HH, HL), each (sh_l, sw_l) with
    missing odd-index entries zero."""
    L = levels(img.shape[1], img.shape[0])
    bands = []
    cur = img.astype(np.float64)
    for _ in range(L):
        h, w = cur.shape
        lo, hi = lift_fwd(cur)                       # rows
        ll, lh = lift_fwd(lo.T)                      # columns of the low half
        hl, hh = lift_fwd(hi.T)
        ll, lh, hl, hh = ll.T, lh.T, hl.T, hh.T
        sh, sw = (h + 1) // 2, (w + 1) // 2

        def pad(a):
            out = np.zeros((sh, sw))
            out[: a.shape[0], : a.shape[1]] = a
            return out
        bands.append((pad(lh), pad(hh), pad(hl)))
        cur = ll
    return bands, cur


def dwt_inverse(bands, lowpass, w: int, h: int) -> np.ndarray:
    dims = []
    cw, ch = w, h
    for _ in bands:
        dims.append((ch, cw))
        cw, ch = (cw + 1) // 2, (ch + 1) // 2
    cur = lowpass
    for l in range(len(bands) - 1, -1, -1):
        hh_, ww_ = dims[l]
        lh, hhb, hl = bands[l]
        ne_r, no_r = (hh_ + 1) // 2, hh_ // 2
        ne_c, no_c = (ww_ + 1) // 2, ww_ // 2
        lo = lift_inv(cur[:ne_r, :ne_c].T, lh[:no_r, :ne_c].T).T     # columns
        hi = lift_inv(hl[:ne_r, :no_c].T, hhb[:no_r, :no_c].T).T
        cur = lift_inv(lo, hi)                                       # rows
    return cur


# ---------------------------------------------------------------- IIR filter
def iir_design(f_low: float, f_high: float, fs: float):
    """FP64 Butterworth HP + LP biquads {b0,b1,b2,a1,a2} x 2 and the warmup."""
    s2 = math.sqrt(2.0)
    wc = math.tan(math.pi * f_low / fs)
    norm = 1.0 / (1.0 + s2 * wc + wc * wc)
    hp = [norm, -2.0 * norm, norm, 2.0 * (wc * wc - 1.0) * norm, (1.0 - s2 * wc + wc * wc) * norm]
    wc = math.tan(math.pi * f_high / fs)
    norm = 1.0 / (1.0 + s2 * wc + wc * wc)
    b0 = wc * wc * norm
    lp = [b0, 2.0 * b0, b0, 2.0 * (wc * wc - 1.0) * norm, (1.0 - s2 * wc + wc * wc) * norm]
    warmup = max(30, int(7.0 * fs / (2.0 * math.pi * f_low)))
    return np.array(hp + lp, dtype=np.float64), warmup


def cascade(c, st, x):
    """One DF-II-transposed step of HP then LP; st = [4, n] (w1, w2 per section)."""
    y = c[0] * x + st[0]
    st[0] = c[1] * x - c[3] * y + st[1]
    st[1] = c[2] * x - c[4] * y
    x = y
    y = c[5] * x + st[2]
    st[2] = c[6] * x - c[8] * y + st[3]
    st[3] = c[7] * x - c[9] * y
    return y


def preseed(c, warmup: int, x: np.ndarray) -> np.ndarray:
    """State after `warmup` cascade steps from zero with the constant input x.
    The cascade is linear and time-invariant, so that state is x times the
    state reached from input 1 (iterated once, on scalars)."""
    one = np.zeros((4, 1))
    for _ in range(warmup):
        cascade(c, one, 1.0)
    return one * np.asarray(x, dtype=np.float64)[None, :]


def fade_amp(amp: float, frames_before: int, warmup: int) -> float:
    g = frames_before - warmup
    if g < 0:
        return 0.0
    if g >= 15:
        return amp
    return ((g + 1) / 15.0) ** 2 * amp


# ------------------------------------------------------ window filter
def window_delta(x: np.ndarray, bilateral: bool) -> np.ndarray:
    """Window-mode delta (temporal_filter.c:170-319) of x = [ws, n], oldest
    sample first: x_c - mean with c = ws / 2, or with bilateral weighting
    w_t = exp(-(x_t - x_c)^2 / (2 s^2)) exp(-(t - c)^2 / (2 (0.15 ws)^2)),
    s = max(0.5 mean |x_t - x_c|, 1e-3): sum w (x - mean) / sum w."""
    x = np.asarray(x, dtype=np.float64)
    ws = x.shape[0]
    c = ws // 2
    mean = x.mean(axis=0)
    cur = x[c]
    d = cur - mean
    if not bilateral:
        return d
    sigma = np.maximum(0.5 * np.abs(x - cur).mean(axis=0), 1e-3)
    t = np.arange(ws, dtype=np.float64)[:, None]
    tw = np.exp(-((t - c) ** 2) / (2.0 * (0.15 * ws) ** 2))
    w = np.exp(-((x - cur) ** 2) / (2.0 * sigma ** 2)) * tw
    sw = w.sum(axis=0)
    res = (w * (x - mean)).sum(axis=0)
    return np.where(sw > 1e-8, res / np.where(sw > 1e-8, sw, 1.0), d)


# ----------------------------------------------------------- guided filter
def box(img: np.ndarray, r: int = 4) -> np.ndarray:
    """radius-r box mean, window clipped at the borders: rows then columns."""
    def along(a, axis):
        n = a.shape[axis]
        z = np.zeros_like(np.take(a, [0], axis=axis))
        c = np.cumsum(np.concatenate([z, a], axis=axis), axis=axis)
        i = np.arange(n)
        lo, hi = np.maximum(i - r, 0), np.minimum(i + r, n - 1) + 1
        s = np.take(c, hi, axis=axis) - np.take(c, lo, axis=axis)
        shape = [1] * a.ndim
        shape[axis] = n
        return s / (hi - lo).reshape(shape)
    return along(along(img, 1), 0)


def guided(I: np.ndarray, p: np.ndarray, r: int = 4, eps: float = 0.01) -> np.ndarray:
    mI, mp = box(I, r), box(p, r)
    cov = box(I * p, r) - mI * mp
    var = box(I * I, r) - mI * mI
    a = cov / (var + eps)
    b = mp - a * mI
    return box(a, r) * I + box(b, r)


def to_u8(v: np.ndarray) -> np.ndarray:
    return np.floor(np.clip(v, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)


class Stream64:
    """IIR luma stream in FP64 (edge-aware guided transfer).  `coef`: use
    these biquad coefficients (e.g. the FP32 design, promoted) instead of the
    FP64 design; process(..., thr=...) overrides the threshold."""

    def __init__(self, width, height, fps=30.0, amp=50.0, f_low=0.5, f_high=3.0, coef=None):
        self.w, self.h, self.amp = width, height, amp
        c, self.warmup = iir_design(f_low, f_high, fps)
        self.c = np.asarray(coef, dtype=np.float64) if coef is not None else c
        self.state = None
        self.frames = 0
        self.last = {}

    def coefficients(self, rgb_u8: np.ndarray):
        """(flat unique detail coefficients, bands, lowpass, guide) of a frame."""
        rgb = rgb_u8.astype(np.float64) / 255.0
        I = gray(rgb)
        bands, low = dwt_forward(I)
        flat = np.concatenate([b.ravel() for lvl in bands for b in lvl])
        return flat, bands, low, I, rgb

    def step(self, flat: np.ndarray) -> np.ndarray:
        """The band-passed delta of one frame's coefficients (preseed first)."""
        if self.state is None:
            self.state = preseed(self.c, self.warmup, flat)
            self.frames = self.warmup
        return cascade(self.c, self.state, flat)

    def process(self, rgb_u8: np.ndarray, thr: float | None = None) -> np.ndarray:
        flat, bands, low, I, rgb = self.coefficients(rgb_u8)
        delta = self.step(flat)
        amp = fade_amp(self.amp, self.frames, self.warmup)
        self.frames += 1
        t = 0.2 * float(np.mean(np.abs(flat))) if thr is None else float(thr)
        out, k = [], 0
        for l, lvl in enumerate(bands):
            a = amp * 0.5 if l == 0 else amp
            nb = []
            for b in lvl:
                d = delta[k: k + b.size].reshape(b.shape)
                nb.append(np.where(np.abs(b) > t, b + a * d, b))
                k += b.size
            out.append(tuple(nb))
        gray_out = dwt_inverse(out, low, self.w, self.h)
        q = guided(I, gray_out - I)
        self.last = {"gray_in": I, "coef": flat, "delta": delta, "thr": t, "gray_out": gray_out}
        return np.clip(rgb + q[..., None], 0.0, 1.0)
