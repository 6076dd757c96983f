/*
 * synth.c - seeded synthetic RGB24 video (see synth.h for the model).
 *
 * Randomness is counter based (a 64-bit finaliser over seed, frame, pixel and
 * channel), so the output does not depend on thread count or frame order.
 * Gaussian samples come from the inverse normal CDF (P. J. Acklam's rational
 * approximation, refined with one Halley step on erfc) tabulated at 65536
 * probability midpoints.
 */
#define _DEFAULT_SOURCE
#include "synth.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TEX 96           /* disc texture grid (covers radius up to 46 px) */
#define NORM_TABLE 65536

struct SynthStream {
    SynthParams p;
    float *bg;           /* [3][H*W] background in LSB units */
    float  tex[3][TEX][TEX];
    float  disc_cx[SYNTH_MAX_DISCS], disc_cy[SYNTH_MAX_DISCS];
    float  disc_dx[SYNTH_MAX_DISCS], disc_dy[SYNTH_MAX_DISCS];
    float  phase[SYNTH_MAX_DISCS];
    float  norm[NORM_TABLE];
};

static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct { uint64_t s; } Rng;
static double rng_u01(Rng *r) {
    r->s = mix64(r->s);
    return (double)(r->s >> 11) * (1.0 / 9007199254740992.0);
}

/* Inverse standard normal CDF (Acklam), refined once with Halley's method. */
static double inv_norm(double p) {
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02,
        -2.759285104469687e+02, 1.383577518672690e+02, -3.066479806614716e+01,
        2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02,
        -1.556989798598866e+02, 6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01,
        -2.400758277161838e+00, -2.549732539343734e+00, 4.374664141464968e+00,
        2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01,
        2.445134137142996e+00, 3.754408661907416e+00};
    const double plow = 0.02425, phigh = 1 - plow;
    double x, q, r;
    if (p < plow) {
        q = sqrt(-2 * log(p));
        x = (((((c[0]*q+c[1])*q+c[2])*q+c[3])*q+c[4])*q+c[5]) /
            ((((d[0]*q+d[1])*q+d[2])*q+d[3])*q+1);
    } else if (p <= phigh) {
        q = p - 0.5; r = q * q;
        x = (((((a[0]*r+a[1])*r+a[2])*r+a[3])*r+a[4])*r+a[5])*q /
            (((((b[0]*r+b[1])*r+b[2])*r+b[3])*r+b[4])*r+1);
    } else {
        q = sqrt(-2 * log(1 - p));
        x = -(((((c[0]*q+c[1])*q+c[2])*q+c[3])*q+c[4])*q+c[5]) /
             ((((d[0]*q+d[1])*q+d[2])*q+d[3])*q+1);
    }
    double e = 0.5 * erfc(-x / sqrt(2.0)) - p;
    double u = e * sqrt(2 * M_PI) * exp(x * x / 2);
    return x - u / (1 + x * u / 2);
}

SynthStream *synth_new(const SynthParams *p) {
    if (p->width < 1 || p->height < 1 || p->n_discs < 0 || p->n_discs > SYNTH_MAX_DISCS)
        return NULL;
    SynthStream *s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->p = *p;
    const int W = p->width, H = p->height;
    const size_t P = (size_t)W * H;
    s->bg = malloc(3 * P * sizeof(float));
    if (!s->bg) { free(s); return NULL; }

    for (int i = 0; i < NORM_TABLE; i++)
        s->norm[i] = (float)inv_norm((i + 0.5) / NORM_TABLE);

    Rng r = { p->seed * 0x2545F4914F6CDD1Dull + 1 };
    /* gradient direction and per-channel tint */
    double gang = 2 * M_PI * rng_u01(&r);
    double gx = cos(gang), gy = sin(gang), tint[3];
    for (int c = 0; c < 3; c++) tint[c] = 0.7 + 0.6 * rng_u01(&r);

    enum { NB = 64 };
    double bx[NB], by[NB], bs[NB], ba[NB][3];
    for (int k = 0; k < NB; k++) {
        bx[k] = rng_u01(&r) * W;
        by[k] = rng_u01(&r) * H;
        bs[k] = 8.0 + 32.0 * rng_u01(&r);
        double lum = 2 * rng_u01(&r) - 1;
        for (int c = 0; c < 3; c++) ba[k][c] = lum + 0.35 * (2 * rng_u01(&r) - 1);
    }
    for (int c = 0; c < 3; c++) {
        float *plane = s->bg + c * P;
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                plane[(size_t)y * W + x] = (float)(tint[c] *
                    (gx * (x - 0.5 * W) / (W + H) + gy * (y - 0.5 * H) / (W + H)));
        for (int k = 0; k < NB; k++) {
            int rad = (int)ceil(4 * bs[k]);
            int x0 = (int)bx[k] - rad, x1 = (int)bx[k] + rad;
            int y0 = (int)by[k] - rad, y1 = (int)by[k] + rad;
            if (x0 < 0) x0 = 0;
            if (y0 < 0) y0 = 0;
            if (x1 > W - 1) x1 = W - 1;
            if (y1 > H - 1) y1 = H - 1;
            double inv = 1.0 / (2 * bs[k] * bs[k]);
            #pragma omp parallel for schedule(static)
            for (int y = y0; y <= y1; y++)
                for (int x = x0; x <= x1; x++) {
                    double dx = x - bx[k], dy = y - by[k];
                    plane[(size_t)y * W + x] += (float)(0.5 * ba[k][c] * exp(-(dx * dx + dy * dy) * inv));
                }
        }
        float lo = plane[0], hi = plane[0];
        for (size_t i = 1; i < P; i++) {
            if (plane[i] < lo) lo = plane[i];
            if (plane[i] > hi) hi = plane[i];
        }
        float scale = (hi > lo) ? 170.0f / (hi - lo) : 0.0f;
        for (size_t i = 0; i < P; i++) plane[i] = 40.0f + (plane[i] - lo) * scale;
    }

    /* disc texture: smooth random field plus a high-contrast stripe pattern */
    for (int c = 0; c < 3; c++) {
        double f1 = 0.15 + 0.3 * rng_u01(&r), f2 = 0.15 + 0.3 * rng_u01(&r);
        double p1 = 2 * M_PI * rng_u01(&r), p2 = 2 * M_PI * rng_u01(&r);
        double base = 60 + 120 * rng_u01(&r);
        for (int v = 0; v < TEX; v++)
            for (int u = 0; u < TEX; u++)
                s->tex[c][v][u] = (float)(base + 45 * sin(f1 * u + p1) * cos(f2 * v + p2)
                                          + 25 * (((u / 6) + (v / 6)) & 1 ? 1 : -1));
    }
    for (int k = 0; k < p->n_discs; k++) {
        double margin = p->disc_radius + 4;
        double spanx = W - 2 * margin, spany = H - 2 * margin;
        s->disc_cx[k] = (float)(margin + (spanx > 0 ? spanx * rng_u01(&r) : 0.5 * W - margin));
        s->disc_cy[k] = (float)(margin + (spany > 0 ? spany * rng_u01(&r) : 0.5 * H - margin));
        double ang = 2 * M_PI * rng_u01(&r);
        s->disc_dx[k] = (float)cos(ang);
        s->disc_dy[k] = (float)sin(ang);
        s->phase[k] = (float)(2 * M_PI * rng_u01(&r));
    }
    return s;
}

void synth_free(SynthStream *s) {
    if (!s) return;
    free(s->bg);
    free(s);
}

static float tex_bilinear(const float t[TEX][TEX], double u, double v) {
    if (u < 0) u = 0;
    if (v < 0) v = 0;
    if (u > TEX - 1.001) u = TEX - 1.001;
    if (v > TEX - 1.001) v = TEX - 1.001;
    int iu = (int)u, iv = (int)v;
    double fu = u - iu, fv = v - iv;
    double a = t[iv][iu] * (1 - fu) + t[iv][iu + 1] * fu;
    double b = t[iv + 1][iu] * (1 - fu) + t[iv + 1][iu + 1] * fu;
    return (float)(a * (1 - fv) + b * fv);
}

void synth_frame(const SynthStream *s, int t, uint8_t *rgb) {
    const SynthParams *p = &s->p;
    const int W = p->width, H = p->height;
    const size_t P = (size_t)W * H;
    const double time = t / (double)p->fps;
    const double flick = p->flicker_amp != 0.0f
        ? p->flicker_amp * sin(2 * M_PI * p->flicker_freq * time) : 0.0;
    double cx[SYNTH_MAX_DISCS], cy[SYNTH_MAX_DISCS];
    for (int k = 0; k < p->n_discs; k++) {
        double d = p->disc_amp[k] * sin(2 * M_PI * p->disc_freq[k] * time + s->phase[k]);
        cx[k] = s->disc_cx[k] + d * s->disc_dx[k];
        cy[k] = s->disc_cy[k] + d * s->disc_dy[k];
    }
    const double R = p->disc_radius;
    const uint64_t fkey = mix64(p->seed ^ ((uint64_t)(uint32_t)t * 0xD6E8FEB86659FD93ull));

    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            size_t i = (size_t)y * W + x;
            float v[3] = { s->bg[i], s->bg[P + i], s->bg[2 * P + i] };
            for (int k = 0; k < p->n_discs; k++) {
                double dx = x - cx[k], dy = y - cy[k];
                if (dx < -R - 1 || dx > R + 1 || dy < -R - 1 || dy > R + 1) continue;
                double cov = R + 0.5 - sqrt(dx * dx + dy * dy);
                if (cov <= 0) continue;
                if (cov > 1) cov = 1;
                double u = dx + 0.5 * TEX, w = dy + 0.5 * TEX;
                for (int c = 0; c < 3; c++)
                    v[c] = (float)((1 - cov) * v[c] + cov * tex_bilinear(s->tex[c], u, w));
            }
            uint64_t h = mix64(fkey ^ (i * 0x9E3779B97F4A7C15ull));
            for (int c = 0; c < 3; c++) {
                uint32_t u16 = (uint32_t)(h >> (16 * c)) & 0xFFFFu;
                double val = v[c] + flick + p->noise_sigma * s->norm[u16];
                long q = lround(val);
                rgb[3 * i + c] = (uint8_t)(q < 0 ? 0 : (q > 255 ? 255 : q));
            }
        }
    }
}

void synth_frames(const SynthStream *s, int t0, int count, uint8_t *rgb) {
    size_t fsz = (size_t)s->p.width * s->p.height * 3;
    for (int k = 0; k < count; k++) synth_frame(s, t0 + k, rgb + (size_t)k * fsz);
}
