/*
 * dropin.c - a C11 caller of the reference API, compiled against include/ and
 * linked with libwema_cuda (tests/test_gpu_dropin.py builds and drives it).
 *
 *   pipeline W H FPS AMP FL FH WS EDGE BIL COLOR IIR BATCH N in out
 *       the reference CLI's call sequence (main.c:278-488): wema_init, flags,
 *       wema_init_color / wema_init_iir / wema_init_iir_color, then the batch
 *       route (IIR luma, BATCH > 1) or wema_process_frame per frame
 *   dwt W H in flat6 low inv      dwt_forward / dwt_inverse
 *   iir N F FL FH FS in out       iir_temporal_* (preseed, single and batch)
 *   amp W H ALPHA orig delta out  coeff_amplify
 *   window W H WS BIL F in out    temporal_buffer_push / temporal_filter_apply
 * Files are raw float32.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dwt.h"
#include "iir_filter.h"
#include "phase_amp.h"
#include "temporal_filter.h"
#include "wema.h"

static float *read_f32(const char *path, size_t n) {
    float *p = malloc(n * sizeof(float));
    FILE *f = fopen(path, "rb");
    if (!p || !f || fread(p, sizeof(float), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return p;
}

static void write_f32(const char *path, const float *p, size_t n) {
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(p, sizeof(float), n, f) != n) {
        fprintf(stderr, "cannot write %s\n", path);
        exit(2);
    }
    fclose(f);
}

static void flatten(const DWTCoeffs *c, float *flat) {
    size_t pos = 0;
    for (int l = 0; l < c->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            size_t n = (size_t)c->subbands[l][o].width * c->subbands[l][o].height;
            memcpy(flat + pos, c->subbands[l][o].coeffs, n * sizeof(float));
            pos += n;
        }
}

static void unflatten(const float *flat, DWTCoeffs *c) {
    size_t pos = 0;
    for (int l = 0; l < c->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            size_t n = (size_t)c->subbands[l][o].width * c->subbands[l][o].height;
            memcpy(c->subbands[l][o].coeffs, flat + pos, n * sizeof(float));
            pos += n;
        }
}

static int pipeline(char **a) {
    int w = atoi(a[0]), h = atoi(a[1]);
    float fps = atof(a[2]), amp = atof(a[3]), fl = atof(a[4]), fh = atof(a[5]);
    int ws = atoi(a[6]), edge = atoi(a[7]), bil = atoi(a[8]), color = atoi(a[9]);
    int iir = atoi(a[10]), batch = atoi(a[11]), nframes = atoi(a[12]);
    size_t fsz = (size_t)w * h * 3;
    float *in = read_f32(a[13], fsz * nframes);
    float *out = malloc(fsz * nframes * sizeof(float));

    WemaContext ctx;
    if (wema_init(&ctx, w, h, fps, amp, fl, fh, ws) < 0) return 3;
    ctx.edge_aware = edge;
    ctx.bilateral_temp = bil;
    ctx.color_mode = color;
    if (color && wema_init_color(&ctx) < 0) return 3;
    if (iir) {
        if (wema_init_iir(&ctx) < 0) return 3;
        if (color && wema_init_iir_color(&ctx) < 0) return 3;
    }
    if (iir && batch > 1 && !color) {
        WemaBatchContext b;
        if (wema_batch_init(&b, &ctx, batch, 0) < 0) return 3;
        Frame *fi = calloc(batch, sizeof(Frame)), *fo = calloc(batch, sizeof(Frame));
        for (int t0 = 0; t0 < nframes; t0 += batch) {
            int cnt = nframes - t0 < batch ? nframes - t0 : batch;
            for (int k = 0; k < cnt; k++) {
                fi[k] = (Frame){in + (t0 + k) * fsz, w, h, 3};
                fo[k] = (Frame){out + (t0 + k) * fsz, w, h, 3};
            }
            if (wema_batch_process(&ctx, &b, fi, fo, cnt) != cnt) return 4;
        }
        wema_batch_free(&b);
        free(fi);
        free(fo);
    } else {
        for (int t = 0; t < nframes; t++) {
            Frame fi = {in + t * fsz, w, h, 3}, fo = {out + t * fsz, w, h, 3};
            if (wema_process_frame(&ctx, &fi, &fo) != 0) return 4;
        }
    }
    Frame dummy = {0};
    if (wema_flush(&ctx, &dummy) != -1) return 5;
    printf("frames_processed %d ready %d\n",
           ctx.iir_filt ? ctx.iir_filt->frames_processed : -1, (int)wema_ready(&ctx));
    write_f32(a[14], out, fsz * nframes);
    wema_free(&ctx);
    return 0;
}

static int dwt(char **a) {
    int w = atoi(a[0]), h = atoi(a[1]);
    float *img = read_f32(a[2], (size_t)w * h);
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return 3;
    dwt_forward(img, w, h, &c);
    size_t n6 = dwt_num_positions(&c);
    float *flat = malloc(n6 * sizeof(float));
    flatten(&c, flat);
    write_f32(a[3], flat, n6);
    write_f32(a[4], c.lowpass, (size_t)c.lowpass_w * c.lowpass_h);
    dwt_inverse(&c, img);
    write_f32(a[5], img, (size_t)w * h);
    dwt_free(&c);
    return 0;
}

static int iir(char **a) {
    size_t n = (size_t)atol(a[0]);
    int frames = atoi(a[1]);
    float *x = read_f32(a[5], n * frames), *y = malloc(n * frames * sizeof(float));
    IIRTemporalFilter f;
    if (iir_temporal_init(&f, n, atof(a[2]), atof(a[3]), atof(a[4])) < 0) return 3;
    iir_temporal_preseed(&f, x);
    if (!iir_temporal_ready(&f)) return 4;
    int half = frames / 2;
    for (int t = 0; t < half; t++) iir_temporal_process(&f, x + t * n, y + t * n);
    iir_temporal_process_batch(&f, x + half * n, y + half * n, frames - half);
    printf("frames_processed %d warmup %d\n", f.frames_processed, f.warmup_frames);
    write_f32(a[6], y, n * frames);
    iir_temporal_free(&f);
    return 0;
}

static int amp(char **a) {
    int w = atoi(a[0]), h = atoi(a[1]);
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return 3;
    size_t n6 = dwt_num_positions(&c);
    float *orig = read_f32(a[3], n6), *delta = read_f32(a[4], n6), *out = malloc(n6 * sizeof(float));
    coeff_amplify(delta, orig, atof(a[2]), &c);
    flatten(&c, out);
    write_f32(a[5], out, n6);
    dwt_free(&c);
    return 0;
}

static int window(char **a) {
    int w = atoi(a[0]), h = atoi(a[1]), ws = atoi(a[2]), bil = atoi(a[3]), frames = atoi(a[4]);
    DWTCoeffs c;
    if (dwt_init(&c, w, h, dwt_compute_levels(w, h)) < 0) return 3;
    size_t n6 = dwt_num_positions(&c);
    float *in = read_f32(a[5], n6 * frames), *out = malloc(n6 * sizeof(float));
    TemporalFilter tf;
    TemporalBuffer tb;
    if (temporal_filter_init(&tf, 0.1f, 0.4f, ws) < 0 || temporal_buffer_init(&tb, &c, ws) < 0) return 3;
    for (int t = 0; t < frames; t++) {
        unflatten(in + t * n6, &c);
        temporal_buffer_push(&tb, &c);
    }
    if (!temporal_buffer_ready(&tb)) return 4;
    temporal_filter_apply(&tf, &tb, out, bil);
    printf("output_count %d head %d\n", temporal_buffer_output_count(&tb), tb.head);
    write_f32(a[6], out, n6);
    temporal_buffer_free(&tb);
    temporal_filter_free(&tf);
    dwt_free(&c);
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 2) return 1;
    if (!strcmp(argv[1], "pipeline") && argc == 17) return pipeline(argv + 2);
    if (!strcmp(argv[1], "dwt") && argc == 8) return dwt(argv + 2);
    if (!strcmp(argv[1], "iir") && argc == 9) return iir(argv + 2);
    if (!strcmp(argv[1], "amp") && argc == 8) return amp(argv + 2);
    if (!strcmp(argv[1], "window") && argc == 9) return window(argv + 2);
    fprintf(stderr, "bad arguments\n");
    return 1;
}
