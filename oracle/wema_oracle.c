/*
 * wema_oracle.c - CPU restatement of the reference's per-frame path (test
 * infrastructure; see wema_oracle.h).  Citations are file:line within the
 * reference project (src/...).
 *
 * How the reference's -Ofast build evaluates each expression was read from
 * GCC's own optimised-tree dump of the reference sources compiled here; the
 * forms are reproduced below with explicit fmaf().  Where GCC vectorised a
 * loop, the vector body and the scalar epilogue can evaluate the same source
 * expression in different orders; vec_cover() gives how many leading elements
 * the vector code handles (an 8-wide body, then at most one 4-wide block).
 */
#define _POSIX_C_SOURCE 200809L
#include "wema_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX_LEVELS 4
#define N_SLOTS 6

/* CDF 9/7 lifting constants (dwt.c:31-36) */
static const float LA = -1.586134342059924f;
static const float LB = -0.052980118572961f;
static const float LG = 0.882911075530934f;
static const float LD = 0.443506852043971f;
static const float LK = 1.149604398860241f;
#define LK_INV (1.0f / 1.149604398860241f)

/* Elements handled by the 8-wide body plus the optional 4-wide block of a
 * GCC-vectorised loop over n elements (scalar code does the rest). */
static long vec_cover(long n) {
    long main = (n - 1 <= 6) ? 0 : (n & ~7L);
    long rem = n - main;
    return main + (rem >= 4 ? 4 : 0);
}

/* ---------------------------------------------------------------- geometry */

int orc_levels(int w, int h) {               /* dwt.c:588-596 */
    int m = w < h ? w : h, l = 0;
    while (m >= 16 && l < MAX_LEVELS) { m /= 2; l++; }
    return l > 0 ? l : 1;
}

int orc_subband_dims(int w, int h, int *sw, int *sh) {   /* dwt.c:608-621 */
    int L = orc_levels(w, h);
    for (int l = 0; l < L; l++) {
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        sw[l] = w;
        sh[l] = h;
    }
    return L;
}

long orc_positions(int w, int h) {           /* dwt.c:769-778 */
    int sw[MAX_LEVELS], sh[MAX_LEVELS];
    int L = orc_subband_dims(w, h, sw, sh);
    long n = 0;
    for (int l = 0; l < L; l++) n += (long)N_SLOTS * sw[l] * sh[l];
    return n;
}

/* ------------------------------------------------------- pixel conversions */

void orc_u8_lut(float *lut) {
    for (int i = 0; i < 256; i++) lut[i] = (float)i / 255.0f;   /* ffmpeg_io.c:293 */
}

void orc_u8_to_float(const uint8_t *src, long n, float *dst) {
    float lut[256];
    orc_u8_lut(lut);
    for (long i = 0; i < n; i++) dst[i] = lut[src[i]];
}

/* clamp to [0,1] then (uint8)(v*255+0.5) (ffmpeg_io.c:305-310), each
 * operation rounded on its own */
void orc_float_to_u8(const float *src, long n, uint8_t *dst) {
    for (long i = 0; i < n; i++) {
        float v = src[i];
        if (v < 0.0f) v = 0.0f;
        if (v > 1.0f) v = 1.0f;
        volatile float t = v * 255.0f;
        dst[i] = (uint8_t)(t + 0.5f);
    }
}

/* Y = .299R+.587G+.114B (wema.c:42-51): vector body
 * fma(b,.114,fma(r,.299,g*.587)), scalar tail fma(r,.299,fma(g,.587,b*.114)) */
static inline float luma_vec(float r, float g, float b) {
    return fmaf(b, 0.114f, fmaf(r, 0.299f, g * 0.587f));
}
static inline float luma_tail(float r, float g, float b) {
    return fmaf(r, 0.299f, fmaf(g, 0.587f, b * 0.114f));
}

void orc_gray(const float *rgb, long n, float *y) {
    long v = vec_cover(n);
    for (long i = 0; i < n; i++) {
        const float *p = rgb + 3 * i;
        y[i] = i < v ? luma_vec(p[0], p[1], p[2]) : luma_tail(p[0], p[1], p[2]);
    }
}

/* BT.601 YCbCr with Cb/Cr + 0.5 (wema.c:60-78) */
void orc_ycbcr(const float *rgb, long n, float *y, float *cb, float *cr) {
    long v = vec_cover(n);
    for (long i = 0; i < n; i++) {
        float r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        if (i < v) {
            y[i] = luma_vec(r, g, b);
            cb[i] = fmaf(-g, 0.331f, 0.5f) + fmaf(r, -0.169f, b * 0.5f);
            cr[i] = fmaf(-b, 0.081f, fmaf(-g, 0.419f, (r + 1.0f) * 0.5f));
        } else {
            y[i] = luma_tail(r, g, b);
            cb[i] = fmaf(-g, 0.331f, b * 0.5f) + fmaf(r, -0.169f, 0.5f);
            cr[i] = fmaf(r + 1.0f, 0.5f, -fmaf(g, 0.419f, b * 0.081f));
        }
    }
}

static inline float clamp01(float v) {        /* MAX(MIN(v,1),0) */
    v = v < 1.0f ? v : 1.0f;
    return v > 0.0f ? v : 0.0f;
}

/* inverse with clamp (wema.c:80-102); same form in body and tail */
void orc_ycbcr_to_rgb(const float *y, const float *cb, const float *cr, long n, float *rgb) {
    for (long i = 0; i < n; i++) {
        float yv = y[i], cbv = cb[i] - 0.5f, crv = cr[i] - 0.5f;
        float r = fmaf(crv, 1.402f, yv);
        float g = yv - fmaf(cbv, 0.344f, crv * 0.714f);
        float b = fmaf(cbv, 1.772f, yv);
        rgb[3 * i] = clamp01(r);
        rgb[3 * i + 1] = clamp01(g);
        rgb[3 * i + 2] = clamp01(b);
    }
}

/* ------------------------------------------------------------- 1D lifting */

/* One predict step: o[j] += c*(e[j] + e[j+1]), the right neighbour mirrored
 * at the end (dwt.c:63-70).  Update step: e[i] += c*(o[i-1] + o[i]) with both
 * ends mirrored (dwt.c:72-80).  GCC contracts both into fma(sum, c, x). */
static void predict(float *o, const float *e, int no, int ne, float c) {
    for (int j = 0; j < no; j++) {
        int r = j + 1 < ne ? j + 1 : ne - 1;
        o[j] = fmaf(e[j] + e[r], c, o[j]);
    }
}
static void update(float *e, const float *o, int ne, int no, float c) {
    for (int i = 0; i < ne; i++) {
        int l = i > 0 ? i - 1 : 0;
        int r = i < no ? i : no - 1;
        e[i] = fmaf(o[l] + o[r], c, e[i]);
    }
}

/* forward 9/7 on v[0..n): output [L (ceil n/2) | H (floor n/2)] (dwt.c:45-107) */
static void lift_fwd(float *v, int n, float *t) {
    if (n < 2) return;
    int ne = (n + 1) / 2, no = n / 2;
    float *e = t, *o = t + ne;
    for (int i = 0; i < no; i++) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
    if (ne > no) e[no] = v[2 * no];
    predict(o, e, no, ne, LA);
    update(e, o, ne, no, LB);
    predict(o, e, no, ne, LG);
    update(e, o, ne, no, LD);
    for (int i = 0; i < ne; i++) v[i] = e[i] * LK_INV;
    for (int i = 0; i < no; i++) v[ne + i] = o[i] * LK;
}

/* inverse (dwt.c:109-170): undo in reverse order with negated constants */
static void lift_inv(float *v, int n, float *t) {
    if (n < 2) return;
    int ne = (n + 1) / 2, no = n / 2;
    float *e = t, *o = t + ne;
    for (int i = 0; i < ne; i++) e[i] = v[i] * LK;
    for (int i = 0; i < no; i++) o[i] = v[ne + i] * LK_INV;
    update(e, o, ne, no, -LD);
    predict(o, e, no, ne, -LG);
    update(e, o, ne, no, -LB);
    predict(o, e, no, ne, -LA);
    for (int i = 0; i < no; i++) { v[2 * i] = e[i]; v[2 * i + 1] = o[i]; }
    if (ne > no) v[2 * no] = e[no];
}

/* Rows and columns are independent lines, so they are split over OpenMP
 * threads; every line's arithmetic is the same whatever the thread count. */
static void lift_rows(float *img, int w, int h, int inverse) {
    #pragma omp parallel if ((long)w * h > 65536)
    {
        float *t = malloc((w + 1) * sizeof(float));
        #pragma omp for schedule(static)
        for (int y = 0; y < h; y++)
            (inverse ? lift_inv : lift_fwd)(img + (long)y * w, w, t);
        free(t);
    }
}

static void lift_cols(float *img, int w, int h, int inverse) {
    #pragma omp parallel if ((long)w * h > 65536)
    {
        float *t = malloc((h + 1) * sizeof(float));
        float *col = malloc((h + 1) * sizeof(float));
        #pragma omp for schedule(static)
        for (int x = 0; x < w; x++) {
            for (int y = 0; y < h; y++) col[y] = img[(long)y * w + x];
            (inverse ? lift_inv : lift_fwd)(col, h, t);
            for (int y = 0; y < h; y++) img[(long)y * w + x] = col[y];
        }
        free(t);
        free(col);
    }
}

/* ------------------------------------------------------------------ 2D DWT */

/* dwt_forward (dwt.c:645-703 with cdf97_2d_forward 369-473).  The level's
 * quadrants are copied into full-size LH/HL/HH scratch planes and the three
 * slots (plus their mirrors 3-5) are copied from those planes; a subband
 * entry that the quadrant does not cover (odd level input) keeps what the
 * scratch plane held at that flat index - the previous level's value, or 0
 * at level 0, where the reference reads uninitialised heap memory. */
int orc_dwt_forward(const float *img, int w, int h, float *flat6, float *lowpass) {
    long P = (long)w * h;
    int L = orc_levels(w, h);
    float *work = malloc(P * sizeof(float));
    float *ll = malloc(P * sizeof(float));
    float *lh = calloc(P, sizeof(float));
    float *hl = calloc(P, sizeof(float));
    float *hh = calloc(P, sizeof(float));
    if (!work || !ll || !lh || !hl || !hh) {
        free(work); free(ll); free(lh); free(hl); free(hh);
        return -1;
    }
    memcpy(work, img, P * sizeof(float));
    int cw = w, ch = h;
    long pos = 0;
    for (int l = 0; l < L; l++) {
        int sw = (cw + 1) / 2, sh = (ch + 1) / 2;
        int nhx = cw - sw, nhy = ch - sh;
        lift_rows(work, cw, ch, 0);
        lift_cols(work, cw, ch, 0);
        for (int y = 0; y < sh; y++)
            for (int x = 0; x < sw; x++) {
                long k = (long)y * sw + x;
                ll[k] = work[(long)y * cw + x];
                if (x < nhx) hl[k] = work[(long)y * cw + sw + x];
                if (y < nhy) lh[k] = work[(long)(sh + y) * cw + x];
                if (x < nhx && y < nhy) hh[k] = work[(long)(sh + y) * cw + sw + x];
            }
        long n = (long)sw * sh;
        memcpy(flat6 + pos + 0 * n, lh, n * sizeof(float));
        memcpy(flat6 + pos + 1 * n, hh, n * sizeof(float));
        memcpy(flat6 + pos + 2 * n, hl, n * sizeof(float));
        memcpy(flat6 + pos + 3 * n, hl, n * sizeof(float));
        memcpy(flat6 + pos + 4 * n, hh, n * sizeof(float));
        memcpy(flat6 + pos + 5 * n, lh, n * sizeof(float));
        pos += 6 * n;
        memcpy(work, ll, n * sizeof(float));
        cw = sw;
        ch = sh;
    }
    memcpy(lowpass, work, (long)cw * ch * sizeof(float));
    free(work); free(ll); free(lh); free(hl); free(hh);
    return 0;
}

/* dwt_inverse (dwt.c:705-767 with cdf97_2d_inverse 475-582): only slots 0-2
 * are read, only over the quadrant each covers; columns then rows. */
int orc_dwt_inverse(const float *flat6, const float *lowpass, int w, int h, float *img) {
    int L = orc_levels(w, h);
    int lw[MAX_LEVELS + 1], lh[MAX_LEVELS + 1];
    lw[0] = w;
    lh[0] = h;
    for (int l = 1; l <= L; l++) { lw[l] = (lw[l - 1] + 1) / 2; lh[l] = (lh[l - 1] + 1) / 2; }
    long off[MAX_LEVELS];
    long pos = 0;
    for (int l = 0; l < L; l++) { off[l] = pos; pos += 6L * lw[l + 1] * lh[l + 1]; }
    long P = (long)w * h;
    float *work = malloc(P * sizeof(float));
    float *out = malloc(P * sizeof(float));
    if (!work || !out) { free(work); free(out); return -1; }
    memcpy(work, lowpass, (long)lw[L] * lh[L] * sizeof(float));
    for (int l = L - 1; l >= 0; l--) {
        int ow = lw[l], oh = lh[l], sw = lw[l + 1], sh = lh[l + 1];
        long n = (long)sw * sh;
        const float *LH = flat6 + off[l], *HH = LH + n, *HL = LH + 2 * n;
        int nhx = ow - sw, nhy = oh - sh;
        memset(out, 0, (long)ow * oh * sizeof(float));
        for (int y = 0; y < sh; y++)
            for (int x = 0; x < sw; x++) {
                long k = (long)y * sw + x;
                out[(long)y * ow + x] = work[k];
                if (x < nhx) out[(long)y * ow + sw + x] = HL[k];
                if (y < nhy) out[(long)(sh + y) * ow + x] = LH[k];
                if (x < nhx && y < nhy) out[(long)(sh + y) * ow + sw + x] = HH[k];
            }
        lift_cols(out, ow, oh, 1);
        lift_rows(out, ow, oh, 1);
        memcpy(work, out, (long)ow * oh * sizeof(float));
    }
    memcpy(img, work, P * sizeof(float));
    free(work); free(out);
    return 0;
}

/* --------------------------------------------------------------------- IIR */

#define PI_F ((float)3.14159265358979323846)

/* iir_design_bandpass order 2 (iir_filter.c:36-101) as GCC evaluates it:
 * high-pass at f_low, low-pass at f_high. */
int orc_iir_design(float f_low, float f_high, float fs, float *c, int *warmup) {
    if (f_low >= f_high || f_low <= 0 || fs * 0.5f <= f_high) return -1;
    const float s2 = 1.41421356237f;
    /* high-pass section (design_highpass_biquad) */
    float wc = tanf((f_low * PI_F) / fs);
    float ws2 = wc * s2;
    float norm = 1.0f / (fmaf(wc, wc, ws2) + 1.0f);
    c[0] = norm;
    c[1] = norm * -2.0f;
    c[2] = norm;
    c[3] = (fmaf(wc, wc, -1.0f) * 2.0f) * norm;
    c[4] = (fmaf(wc, wc, 1.0f) - ws2) * norm;
    /* low-pass section (design_lowpass_biquad) */
    wc = tanf((f_high * PI_F) / fs);
    float wc2 = wc * wc;
    norm = 1.0f / (fmaf(wc, s2, wc2) + 1.0f);
    c[5] = wc2 * norm;
    c[6] = c[5] * 2.0f;
    c[7] = c[5];
    c[8] = ((wc2 - 1.0f) * 2.0f) * norm;
    c[9] = norm * fmaf(-wc, s2, wc2 + 1.0f);
    /* iir_filter.c:150-151 */
    int wu = (int)(7.0f * fs / (2.0f * PI_F * f_low));
    *warmup = wu < 30 ? 30 : wu;
    return 0;
}

/* one DF-II-transposed cascade step as the AVX-512 path writes it
 * (iir_filter.c:210-224); positions past the last full 16-wide block take the
 * scalar remainder loop, which GCC contracts differently for w2
 * (iir_filter.c:231-246: w2 = fms(b2, x, a2*y)). */
static inline float biquad2(const float *c, float *st, float x, int tail) {
    for (int s = 0; s < 2; s++) {
        const float *k = c + 5 * s;
        float w1 = st[2 * s], w2 = st[2 * s + 1];
        float y = fmaf(k[0], x, w1);
        st[2 * s] = fmaf(-k[3], y, fmaf(k[1], x, w2));
        st[2 * s + 1] = tail ? fmaf(k[2], x, -(k[4] * y)) : fmaf(-k[4], y, k[2] * x);
        x = y;
    }
    return x;
}

void orc_iir_preseed(const float *c, int warmup, const float *x, long n, float *state4) {
    long simd = n & ~15L;                       /* iir_filter.c:376-471 */
    #pragma omp parallel for schedule(static) if (n > 65536)
    for (long i = 0; i < n; i++)
        for (int it = 0; it < warmup; it++) biquad2(c, state4 + 4 * i, x[i], i >= simd);
}

void orc_iir_step(const float *c, const float *x, long n, float *state4, float *out) {
    long simd = n & ~15L;
    #pragma omp parallel for schedule(static) if (n > 65536)
    for (long i = 0; i < n; i++) out[i] = biquad2(c, state4 + 4 * i, x[i], i >= simd);
}

/* ------------------------------------------------- threshold, amplification */

/* sum of |x| as GCC vectorises it (phase_amp.c:25-28, wema.c:719-722,
 * wema_batch.c:272-275): eight running lane sums over the first n&~7
 * elements, reduced ((l0+l4)+(l2+l6))+((l1+l5)+(l3+l7)); a remainder of 4-7
 * first adds four more elements to the half-reduced lanes (l_j+l_{j+4}) and
 * reduces those as (v0+v2)+(v1+v3); what is left is added one by one. */
float orc_mag_sum(const float *x, long n) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float half[4] = {0, 0, 0, 0};
    long i = 0;
    float s = 0.0f;
    if (n - 1 > 6) {
        long m = n & ~7L;
        for (; i < m; i += 8)
            for (int j = 0; j < 8; j++) acc[j] += fabsf(x[i + j]);
        for (int j = 0; j < 4; j++) half[j] = acc[j] + acc[j + 4];
        s = (half[0] + half[2]) + (half[1] + half[3]);
    }
    if (n - i >= 4) {
        float v[4];
        for (int j = 0; j < 4; j++) v[j] = half[j] + fabsf(x[i + j]);
        s = (v[0] + v[2]) + (v[1] + v[3]);
        i += 4;
    }
    for (; i < n; i++) s += fabsf(x[i]);
    return s;
}

/* single-frame route: (sum / N) * 0.2 (wema.c:723, phase_amp.c:29);
 * batch route: (0.2 / N) * sum (wema_batch.c:276, reciprocal hoisted) */
float orc_threshold(const float *orig6, long n, int batch_form) {
    float s = orc_mag_sum(orig6, n);
    if (batch_form) return (0.2f / (float)n) * s;
    return (s / (float)n) * 0.2f;
}

/* out = |orig| > thr ? fma(delta, alpha_l, orig) : orig, alpha_0 = amp/2
 * (wema.c:726-743, phase_amp.c:32-55, wema_batch.c:279-296) */
void orc_amplify(const float *delta6, const float *orig6, float amp, float thr,
                 int w, int h, float *out6) {
    int sw[MAX_LEVELS], sh[MAX_LEVELS];
    int L = orc_subband_dims(w, h, sw, sh);
    long pos = 0;
    for (int l = 0; l < L; l++) {
        float al = l == 0 ? amp * 0.5f : amp;
        long n = 6L * sw[l] * sh[l];
        for (long i = 0; i < n; i++, pos++) {
            float o = orig6[pos];
            out6[pos] = fabsf(o) > thr ? fmaf(delta6[pos], al, o) : o;
        }
    }
}

/* 15-frame quadratic fade-in after the preseed (wema.c:831-839,
 * wema_batch.c:426-435): t = (g+1) * (1/15), amp = (t*t) * amp_factor */
float orc_fade_amp(float amp_factor, int frames_before, int warmup) {
    int g = frames_before - warmup;
    if (g < 0) return 0.0f;
    if (g >= 15) return amp_factor;
    float t = (float)(g + 1) * (1.0f / 15.0f);
    return (t * t) * amp_factor;
}

/* ------------------------------------------------ spatial filters, transfer */

/* radius-r box mean with the window clipped at the borders, evaluated as the
 * reference does: sequential FP32 prefix sums per row, then per column of the
 * row means (wema.c:114-171, wema_batch.c:26-61) */
void orc_box(const float *in, float *out, int w, int h, int r) {
    long P = (long)w * h;
    int md = w > h ? w : h;
    float *tmp = malloc(P * sizeof(float));
    #pragma omp parallel if (P > 65536)
    {
        float *pre = malloc((md + 1) * sizeof(float));
        #pragma omp for schedule(static)
        for (int y = 0; y < h; y++) {
            const float *row = in + (long)y * w;
            pre[0] = 0.0f;
            for (int x = 0; x < w; x++) pre[x + 1] = pre[x] + row[x];
            for (int x = 0; x < w; x++) {
                int a = x - r > 0 ? x - r : 0, b = x + r + 1 < w ? x + r + 1 : w;
                tmp[(long)y * w + x] = (pre[b] - pre[a]) / (float)(b - a);
            }
        }
        #pragma omp for schedule(static)
        for (int x = 0; x < w; x++) {
            pre[0] = 0.0f;
            for (int y = 0; y < h; y++) pre[y + 1] = pre[y] + tmp[(long)y * w + x];
            for (int y = 0; y < h; y++) {
                int a = y - r > 0 ? y - r : 0, b = y + r + 1 < h ? y + r + 1 : h;
                out[(long)y * w + x] = (pre[b] - pre[a]) / (float)(b - a);
            }
        }
        free(pre);
    }
    free(tmp);
}

/* guided filter, output = mean_a*I + mean_b (wema.c:173-230) with GCC's
 * contractions: a = (corr_Ip - mI*mp) / ((corr_I + eps) - mI*mI),
 * b = mp - a*mI */
void orc_guided(const float *I, const float *p, float *out, int w, int h, int r, float eps) {
    long n = (long)w * h;
    float *mI = malloc(n * 4), *mp = malloc(n * 4), *cI = malloc(n * 4), *cIp = malloc(n * 4);
    orc_box(I, mI, w, h, r);
    orc_box(p, mp, w, h, r);
    for (long i = 0; i < n; i++) cI[i] = I[i] * I[i];
    orc_box(cI, cI, w, h, r);
    for (long i = 0; i < n; i++) cIp[i] = I[i] * p[i];
    orc_box(cIp, cIp, w, h, r);
    for (long i = 0; i < n; i++) {
        float a = fmaf(-mI[i], mp[i], cIp[i]) / fmaf(-mI[i], mI[i], cI[i] + eps);
        cI[i] = a;
        cIp[i] = fmaf(-a, mI[i], mp[i]);
    }
    orc_box(cI, mI, w, h, r);
    orc_box(cIp, mp, w, h, r);
    for (long i = 0; i < n; i++) out[i] = fmaf(mI[i], I[i], mp[i]);
    free(mI); free(mp); free(cI); free(cIp);
}

/* separable [1 4 6 4 1]/16 with the weights renormalised at the borders
 * (wema.c:236-283) */
void orc_gauss5(const float *in, float *out, int w, int h) {
    static const float k[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};
    float *tmp = malloc((long)w * h * sizeof(float));
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float s = 0.0f, wt = 0.0f;
            for (int d = -2; d <= 2; d++) {
                int xx = x + d;
                if (xx >= 0 && xx < w) { s = fmaf(in[(long)y * w + xx], k[d + 2], s); wt += k[d + 2]; }
            }
            tmp[(long)y * w + x] = s / wt;
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float s = 0.0f, wt = 0.0f;
            for (int d = -2; d <= 2; d++) {
                int yy = y + d;
                if (yy >= 0 && yy < h) { s = fmaf(tmp[(long)yy * w + x], k[d + 2], s); wt += k[d + 2]; }
            }
            out[(long)y * w + x] = s / wt;
        }
    free(tmp);
}

/* frame_gray_to_rgb_ex (wema.c:289-335) and gray_to_rgb_edge_aware
 * (wema_batch.c:311-346): guide = luma of the input, smooth (gray - guide)
 * with the guided filter (r 4, eps 0.01) or the 5-tap Gaussian, add to RGB,
 * clamp to [0,1]. */
void orc_gray_to_rgb(const float *gray, const float *rgb, int w, int h, int edge_aware,
                     float *out) {
    long n = (long)w * h;
    float *guide = malloc(n * 4), *delta = malloc(n * 4), *smooth = malloc(n * 4);
    long v = vec_cover(n);
    for (long i = 0; i < n; i++) {
        const float *p = rgb + 3 * i;
        guide[i] = i < v ? luma_vec(p[0], p[1], p[2]) : luma_tail(p[0], p[1], p[2]);
        delta[i] = gray[i] - guide[i];
    }
    if (edge_aware) orc_guided(guide, delta, smooth, w, h, 4, 0.01f);
    else orc_gauss5(delta, smooth, w, h);
    for (long i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) {
            float d = rgb[3 * i + c] + smooth[i];
            if (d < 0.0f) d = 0.0f;
            if (d > 1.0f) d = 1.0f;
            out[3 * i + c] = d;
        }
    free(guide); free(delta); free(smooth);
}

/* ------------------------------------------------- window temporal filter */

/* mean-removed centre sample, optionally bilateral-weighted
 * (temporal_filter.c:170-319).  The window starts at the oldest sample
 * (index head), centre = ws/2. */
void orc_window_apply(const float *ring, long n, int ws, int head, int bilateral, float *delta) {
    const int center = ws / 2;
    const float inv_ws = 1.0f / (float)ws;
    float tw[256];
    if (bilateral) {
        float ts = (float)ws * 0.15f;
        float inv2 = 0.5f / (ts * ts);
        for (int t = 0; t < ws; t++) {
            float d = (float)(t - center);
            tw[t] = expf(-(d * d) * inv2);
        }
    }
    #pragma omp parallel for schedule(static) if (n > 16384)
    for (long pos = 0; pos < n; pos++) {
        float raw[256], tmp[256];
        const float *b = ring + pos * ws;
        float mean = 0.0f;
        for (int t = 0; t < ws; t++) {
            raw[t] = b[(head + t) % ws];
            mean += raw[t];
        }
        float cur = raw[center];
        mean = mean * inv_ws;
        for (int t = 0; t < ws; t++) tmp[t] = raw[t] - mean;
        if (!bilateral) { delta[pos] = tmp[center]; continue; }
        float mad = 0.0f;
        for (int t = 0; t < ws; t++) mad += fabsf(raw[t] - cur);
        float sigma = fmaxf((inv_ws * 0.5f) * mad, 0.001f);
        float inv2 = 0.5f / (sigma * sigma);
        float wsum = 0.0f, res = 0.0f, wt[256];
        for (int t = 0; t < ws; t++) {
            float d = raw[t] - cur;
            wt[t] = expf(-(d * d) * inv2) * tw[t];
            wsum += wt[t];
        }
        if (wsum > 1e-8f) {
            for (int t = 0; t < ws; t++) res = fmaf(wt[t], tmp[t], res);
            delta[pos] = res * (1.0f / wsum);
        } else {
            delta[pos] = tmp[center];
        }
    }
}

/* ------------------------------------------------------------ stream driver */

typedef struct {
    float *prev, *delta, *amp6, *state, *lowpass, *out;   /* per channel */
    float *ring, *amplitude;
} Chan;

typedef struct {
    OrcConfig cfg;
    int L, nch, warmup, frames_processed, head, filled;
    long P, N, nlow;
    float coef[10];
    Chan ch[3];
    float *plane[3];      /* Y / Cb / Cr input planes */
} Stream;

void *orc_stream_new(const OrcConfig *cfg) {
    Stream *s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->cfg = *cfg;
    s->L = orc_levels(cfg->width, cfg->height);
    s->P = (long)cfg->width * cfg->height;
    s->N = orc_positions(cfg->width, cfg->height);
    int sw[MAX_LEVELS], sh[MAX_LEVELS];
    orc_subband_dims(cfg->width, cfg->height, sw, sh);
    s->nlow = (long)sw[s->L - 1] * sh[s->L - 1];
    s->nch = cfg->color ? 3 : 1;
    if (cfg->use_iir && orc_iir_design(cfg->f_low, cfg->f_high, cfg->fps, s->coef, &s->warmup) < 0) {
        free(s);
        return NULL;
    }
    for (int c = 0; c < s->nch; c++) {
        Chan *h = &s->ch[c];
        h->prev = calloc(s->N, 4);
        h->delta = calloc(s->N, 4);
        h->amp6 = calloc(s->N, 4);
        h->lowpass = calloc(s->nlow, 4);
        h->out = calloc(s->P, 4);
        if (cfg->use_iir) h->state = calloc(4 * s->N, 4);
        else {
            h->ring = calloc(s->N * (long)cfg->window, 4);
            h->amplitude = calloc(s->N, 4);
        }
        s->plane[c] = calloc(s->P, 4);
    }
    return s;
}

void orc_stream_free(void *p) {
    Stream *s = p;
    if (!s) return;
    for (int c = 0; c < 3; c++) {
        Chan *h = &s->ch[c];
        free(h->prev); free(h->delta); free(h->amp6); free(h->state);
        free(h->lowpass); free(h->out); free(h->ring); free(h->amplitude);
        free(s->plane[c]);
    }
    free(s);
}

int orc_stream_frames_processed(void *p) { return ((Stream *)p)->frames_processed; }

/* wema_process_frame (wema.c:746-952) */
int orc_stream_process(void *p, const float *in, float *out) {
    Stream *s = p;
    const OrcConfig *c = &s->cfg;
    const int W = c->width, H = c->height;
    if (s->nch == 3) orc_ycbcr(in, s->P, s->plane[0], s->plane[1], s->plane[2]);
    else orc_gray(in, s->P, s->plane[0]);
    for (int k = 0; k < s->nch; k++)
        orc_dwt_forward(s->plane[k], W, H, s->ch[k].prev, s->ch[k].lowpass);

    if (c->use_iir) {
        if (s->frames_processed == 0) {
            for (int k = 0; k < s->nch; k++)
                orc_iir_preseed(s->coef, s->warmup, s->ch[k].prev, s->N, s->ch[k].state);
            s->frames_processed = s->warmup;
        }
        int before = s->frames_processed;
        for (int k = 0; k < s->nch; k++)
            orc_iir_step(s->coef, s->ch[k].prev, s->N, s->ch[k].state, s->ch[k].delta);
        s->frames_processed++;
        float amp = orc_fade_amp(c->amp, before, s->warmup);
        for (int k = 0; k < s->nch; k++) {
            Chan *h = &s->ch[k];
            float a = k == 0 ? amp : amp * 0.5f;
            orc_amplify(h->delta, h->prev, a, orc_threshold(h->prev, s->N, 0), W, H, h->amp6);
        }
    } else {
        for (int k = 0; k < s->nch; k++) {           /* temporal_buffer_push */
            Chan *h = &s->ch[k];
            for (long i = 0; i < s->N; i++) {
                h->ring[i * c->window + s->head] = h->prev[i];
                h->amplitude[i] = h->prev[i];
            }
        }
        s->head = (s->head + 1) % c->window;
        if (s->filled < c->window) s->filled++;
        if (s->filled < c->window) {
            memcpy(out, in, (size_t)s->P * 3 * sizeof(float));
            return 0;
        }
        for (int k = 0; k < s->nch; k++) {
            Chan *h = &s->ch[k];
            orc_window_apply(h->ring, s->N, c->window, s->head, c->bilateral, h->delta);
            float a = k == 0 ? c->amp : c->amp * 0.5f;
            orc_amplify(h->delta, h->amplitude, a, orc_threshold(h->amplitude, s->N, 0), W, H, h->amp6);
        }
    }
    for (int k = 0; k < s->nch; k++)
        orc_dwt_inverse(s->ch[k].amp6, s->ch[k].lowpass, W, H, s->ch[k].out);
    if (s->nch == 3) orc_ycbcr_to_rgb(s->ch[0].out, s->ch[1].out, s->ch[2].out, s->P, out);
    else orc_gray_to_rgb(s->ch[0].out, in, W, H, c->edge_aware, out);
    return 0;
}

/* wema_batch_process (wema_batch.c:352-457): IIR luma only, always the
 * guided filter, threshold in the batch form.  Frames are independent except
 * for the IIR state, so a frame-by-frame loop gives the same result. */
int orc_stream_batch(void *p, const float *in, float *out, int count) {
    Stream *s = p;
    const OrcConfig *c = &s->cfg;
    if (!c->use_iir) return -1;
    const int W = c->width, H = c->height;
    Chan *h = &s->ch[0];
    for (int f = 0; f < count; f++) {
        const float *fi = in + (size_t)f * s->P * 3;
        float *fo = out + (size_t)f * s->P * 3;
        orc_gray(fi, s->P, s->plane[0]);
        orc_dwt_forward(s->plane[0], W, H, h->prev, h->lowpass);
        if (s->frames_processed == 0) {
            orc_iir_preseed(s->coef, s->warmup, h->prev, s->N, h->state);
            s->frames_processed = s->warmup;
        }
        float amp = orc_fade_amp(c->amp, s->frames_processed, s->warmup);
        orc_iir_step(s->coef, h->prev, s->N, h->state, h->delta);
        s->frames_processed++;
        orc_amplify(h->delta, h->prev, amp, orc_threshold(h->prev, s->N, 1), W, H, h->amp6);
        orc_dwt_inverse(h->amp6, h->lowpass, W, H, h->out);
        orc_gray_to_rgb(h->out, fi, W, H, 1, fo);
    }
    return count;
}

/* same codes as the reference harness (oracle/ref_harness.c) */
long orc_stream_get(void *p, int what, float *dst) {
    Stream *s = p;
    long n;
    switch (what) {
    case 0: memcpy(dst, s->plane[0], s->P * 4); return s->P;
    case 1: memcpy(dst, s->ch[0].out, s->P * 4); return s->P;
    case 2: n = s->N; memcpy(dst, s->ch[0].prev, n * 4); return n;
    case 3: memcpy(dst, s->ch[0].delta, s->N * 4); return s->N;
    case 4: memcpy(dst, s->ch[0].amp6, s->N * 4); return s->N;
    case 5: memcpy(dst, s->ch[0].lowpass, s->nlow * 4); return s->nlow;
    case 6: if (!s->ch[0].amplitude) return -1; memcpy(dst, s->ch[0].amplitude, s->N * 4); return s->N;
    case 7: if (s->nch < 3) return -1; memcpy(dst, s->ch[1].prev, s->N * 4); return s->N;
    case 8: if (s->nch < 3) return -1; memcpy(dst, s->ch[2].prev, s->N * 4); return s->N;
    case 9: if (s->nch < 3) return -1; memcpy(dst, s->ch[1].delta, s->N * 4); return s->N;
    case 10: if (s->nch < 3) return -1; memcpy(dst, s->ch[2].delta, s->N * 4); return s->N;
    default: return -1;
    }
}
