/*
 * ref_harness.c - drives the UNMODIFIED reference library (built from the
 * reference's own src/*.c into oracle/_ref/) through its public C API, on
 * in-memory frames, so tests and the CPU baseline can call it with flat
 * buffers.  Test infrastructure only: nothing in the product links this.
 *
 * Reference entry points exercised (paths within the reference project):
 *   wema_init / wema_init_color / wema_init_iir / wema_init_iir_color /
 *   wema_process_frame / wema_free            src/wema.c:359-952
 *   wema_batch_init / wema_batch_process       src/wema_batch.c:138-457
 *   dwt_init / dwt_forward / dwt_inverse       src/dwt.c:598-767
 *   iir_design_bandpass / iir_temporal_*       src/iir_filter.c:70-471
 *   coeff_amplify                              src/phase_amp.c:12-56
 *   frame_rgb_to_gray / frame_gray_to_rgb_ex   src/wema.c:42-51, 289-335
 *   temporal_buffer_* / temporal_filter_apply  src/temporal_filter.c:97-319
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#include "wema.h"
#include "dwt.h"
#include "iir_filter.h"
#include "temporal_filter.h"
#include "phase_amp.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* frame_gray_to_rgb_ex is defined non-static in wema.c but not declared in
 * any reference header; declare it here to call it. */
void frame_gray_to_rgb_ex(const float *gray, const Frame *orig, Frame *out,
                          float *delta_buf, float *smooth_buf,
                          float *guide_buf, float *work1, float *work2,
                          float *work3, float *work4, bool edge_aware);

typedef struct {
    int   width, height;
    float fps, amp, f_low, f_high;
    int   window;
    int   edge_aware, bilateral, color, use_iir;
} RhConfig;

typedef struct {
    WemaContext ctx;
    WemaBatchContext batch;
    int has_batch;
    Frame in, out;
    Frame *bin, *bout;
    int batch_size;
} RhStream;

int rh_levels(int w, int h) { return dwt_compute_levels(w, h); }

long rh_num_positions(int w, int h) {
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return -1;
    long n = (long)dwt_num_positions(&c);
    dwt_free(&c);
    return n;
}

static void flatten(const DWTCoeffs *c, float *flat6) {
    size_t pos = 0;
    for (int l = 0; l < c->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            size_t n = (size_t)c->subbands[l][o].width * c->subbands[l][o].height;
            memcpy(flat6 + pos, c->subbands[l][o].coeffs, n * sizeof(float));
            pos += n;
        }
}

static void unflatten(const float *flat6, DWTCoeffs *c) {
    size_t pos = 0;
    for (int l = 0; l < c->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            size_t n = (size_t)c->subbands[l][o].width * c->subbands[l][o].height;
            memcpy(c->subbands[l][o].coeffs, flat6 + pos, n * sizeof(float));
            pos += n;
        }
}

void rh_gray(const float *rgb, int w, int h, float *gray) {
    Frame f = { (float *)rgb, w, h, 3 };
    frame_rgb_to_gray(&f, gray);
}

int rh_dwt_forward(const float *img, int w, int h, float *flat6, float *lowpass) {
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return -1;
    dwt_forward(img, w, h, &c);
    flatten(&c, flat6);
    memcpy(lowpass, c.lowpass, (size_t)c.lowpass_w * c.lowpass_h * sizeof(float));
    dwt_free(&c);
    return 0;
}

int rh_dwt_inverse(const float *flat6, const float *lowpass, int w, int h, float *img) {
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return -1;
    unflatten(flat6, &c);
    memcpy(c.lowpass, lowpass, (size_t)c.lowpass_w * c.lowpass_h * sizeof(float));
    dwt_inverse(&c, img);
    dwt_free(&c);
    return 0;
}

/* coeff_amplify (phase_amp.c) on a flat 6-slot array; writes the amplified
 * 6-slot array. */
int rh_coeff_amplify(const float *delta6, const float *orig6, float alpha,
                     int w, int h, float *out6) {
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return -1;
    coeff_amplify(delta6, orig6, alpha, &c);
    flatten(&c, out6);
    dwt_free(&c);
    return 0;
}

int rh_iir_design(float fl, float fh, float fs, float *coef10, int *warmup) {
    IIRTemporalFilter f;
    int rc = iir_temporal_init(&f, 16, fl, fh, fs);
    if (rc < 0) return rc;
    for (int s = 0; s < 2; s++) {
        coef10[5 * s + 0] = f.coeffs.sections[s].b0;
        coef10[5 * s + 1] = f.coeffs.sections[s].b1;
        coef10[5 * s + 2] = f.coeffs.sections[s].b2;
        coef10[5 * s + 3] = f.coeffs.sections[s].a1;
        coef10[5 * s + 4] = f.coeffs.sections[s].a2;
    }
    *warmup = f.warmup_frames;
    iir_temporal_free(&f);
    return 0;
}

/* Runs nframes frames of n positions through a fresh IIR filter.
 * preseed != 0 preseeds with frame 0 first; batch != 0 uses the batch routine
 * for all frames at once. out is [nframes][n]. */
int rh_iir_run(const float *x, long n, int nframes, float fl, float fh, float fs,
               int preseed, int batch, float *out) {
    IIRTemporalFilter f;
    if (iir_temporal_init(&f, (size_t)n, fl, fh, fs) < 0) return -1;
    if (preseed) iir_temporal_preseed(&f, x);
    if (batch) {
        iir_temporal_process_batch(&f, x, out, nframes);
    } else {
        for (int t = 0; t < nframes; t++)
            iir_temporal_process(&f, x + (size_t)t * n, out + (size_t)t * n);
    }
    iir_temporal_free(&f);
    return 0;
}

/* frame_gray_to_rgb_ex (guided filter or Gaussian fallback + RGB add/clamp). */
int rh_gray_to_rgb(const float *gray, const float *rgb, int w, int h,
                   int edge_aware, float *out_rgb) {
    size_t n = (size_t)w * h;
    float *buf = malloc(n * 7 * sizeof(float));
    if (!buf) return -1;
    Frame orig = { (float *)rgb, w, h, 3 };
    Frame out = { out_rgb, w, h, 3 };
    frame_gray_to_rgb_ex(gray, &orig, &out, buf, buf + n, buf + 2 * n,
                         buf + 3 * n, buf + 4 * n, buf + 5 * n,
                         buf + 6 * n, edge_aware != 0);
    free(buf);
    return 0;
}

/* --- whole-pipeline streams -------------------------------------------- */

void *rh_stream_new(const RhConfig *cfg, int batch_size, int threads) {
    RhStream *s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    if (wema_init(&s->ctx, cfg->width, cfg->height, cfg->fps, cfg->amp,
                  cfg->f_low, cfg->f_high, cfg->window) < 0) { free(s); return NULL; }
    s->ctx.edge_aware = cfg->edge_aware != 0;
    s->ctx.bilateral_temp = cfg->bilateral != 0;
    s->ctx.color_mode = cfg->color != 0;
    if (cfg->color && wema_init_color(&s->ctx) < 0) goto fail;
    if (cfg->use_iir) {
        if (wema_init_iir(&s->ctx) < 0) goto fail;
        if (cfg->color && wema_init_iir_color(&s->ctx) < 0) goto fail;
    }
    if (batch_size > 0) {
        if (wema_batch_init(&s->batch, &s->ctx, batch_size, threads) < 0) goto fail;
        s->has_batch = 1;
        s->batch_size = s->batch.batch_size;
        s->bin = calloc((size_t)s->batch_size, sizeof(Frame));
        s->bout = calloc((size_t)s->batch_size, sizeof(Frame));
    }
    return s;
fail:
    wema_free(&s->ctx);
    free(s);
    return NULL;
}

void rh_stream_free(void *p) {
    RhStream *s = p;
    if (!s) return;
    if (s->has_batch) wema_batch_free(&s->batch);
    free(s->bin);
    free(s->bout);
    wema_free(&s->ctx);
    free(s);
}

int rh_stream_process(void *p, const float *rgb_in, float *rgb_out) {
    RhStream *s = p;
    Frame in = { (float *)rgb_in, s->ctx.width, s->ctx.height, 3 };
    Frame out = { rgb_out, s->ctx.width, s->ctx.height, 3 };
    return wema_process_frame(&s->ctx, &in, &out);
}

int rh_batch_process(void *p, const float *rgb_in, float *rgb_out, int count) {
    RhStream *s = p;
    if (!s->has_batch) return -1;
    size_t fsz = (size_t)s->ctx.width * s->ctx.height * 3;
    if (count > s->batch_size) count = s->batch_size;
    for (int i = 0; i < count; i++) {
        s->bin[i] = (Frame){ (float *)rgb_in + i * fsz, s->ctx.width, s->ctx.height, 3 };
        s->bout[i] = (Frame){ rgb_out + i * fsz, s->ctx.width, s->ctx.height, 3 };
    }
    return wema_batch_process(&s->ctx, &s->batch, s->bin, s->bout, count);
}

/* Copies an internal buffer of the last processed frame:
 * 0 gray_in [P], 1 gray_out [P], 2 prev_coeffs (orig, 6-slot) [N6],
 * 3 delta_phi [N6], 4 amplified 6-slot coefficients [N6], 5 lowpass,
 * 6 temporal amplitude (window mode) [N6], 7 cb prev, 8 cr prev,
 * 9 delta_cb, 10 delta_cr.  Returns the element count copied or -1. */
long rh_stream_get(void *p, int what, float *dst) {
    RhStream *s = p;
    WemaContext *c = &s->ctx;
    size_t P = (size_t)c->width * c->height;
    size_t N = dwt_num_positions(c->coeffs);
    switch (what) {
    case 0: memcpy(dst, c->gray_in, P * 4); return (long)P;
    case 1: memcpy(dst, c->gray_out, P * 4); return (long)P;
    case 2: if (!c->prev_coeffs) return -1; memcpy(dst, c->prev_coeffs, N * 4); return (long)N;
    case 3: memcpy(dst, c->delta_phi, N * 4); return (long)N;
    case 4: flatten(c->coeffs, dst); return (long)N;
    case 5: memcpy(dst, c->coeffs->lowpass, (size_t)c->coeffs->lowpass_w * c->coeffs->lowpass_h * 4);
            return (long)c->coeffs->lowpass_w * c->coeffs->lowpass_h;
    case 6: if (!c->temporal_buf) return -1; memcpy(dst, c->temporal_buf->amplitude, N * 4); return (long)N;
    case 7: if (!c->prev_coeffs_cb) return -1; memcpy(dst, c->prev_coeffs_cb, N * 4); return (long)N;
    case 8: if (!c->prev_coeffs_cr) return -1; memcpy(dst, c->prev_coeffs_cr, N * 4); return (long)N;
    case 9: if (!c->delta_cb) return -1; memcpy(dst, c->delta_cb, N * 4); return (long)N;
    case 10: if (!c->delta_cr) return -1; memcpy(dst, c->delta_cr, N * 4); return (long)N;
    default: return -1;
    }
}

int rh_frames_processed(void *p) {
    RhStream *s = p;
    return s->ctx.iir_filt ? s->ctx.iir_filt->frames_processed : -1;
}

int rh_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}
