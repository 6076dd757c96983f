/*
 * wema_oracle.h - CPU restatement of the reference's per-frame amplification
 * path, used ONLY as the checker by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  It is never linked into libwema_cuda.
 *
 * Every function reproduces the reference's FP32 arithmetic as the reference
 * Makefile's `all` build (gcc -Ofast) evaluates it: the FMA contractions,
 * reassociations and the 8-lane vectorised reductions are written out
 * explicitly with fmaf() so this file is compiled WITHOUT fast-math and gives
 * the same bits on any host.  Parity with the compiled reference is pinned by
 * tests/test_oracle_pin.py.
 */
#ifndef WEMA_ORACLE_H
#define WEMA_ORACLE_H

#include <stdint.h>

/* geometry (dwt.c:588-632) */
int   orc_levels(int w, int h);
long  orc_positions(int w, int h);          /* 6-slot count N6 (dwt.c:769-778) */
int   orc_subband_dims(int w, int h, int *sw, int *sh);   /* returns levels */

/* pixel conversions */
void  orc_u8_lut(float *lut256);
void  orc_u8_to_float(const uint8_t *src, long n, float *dst);
void  orc_float_to_u8(const float *src, long n, uint8_t *dst);
void  orc_gray(const float *rgb, long npix, float *y);
void  orc_ycbcr(const float *rgb, long npix, float *y, float *cb, float *cr);
void  orc_ycbcr_to_rgb(const float *y, const float *cb, const float *cr, long npix, float *rgb);

/* 2D CDF 9/7 DWT; flat6 in the reference's 6-slot flat order */
int   orc_dwt_forward(const float *img, int w, int h, float *flat6, float *lowpass);
int   orc_dwt_inverse(const float *flat6, const float *lowpass, int w, int h, float *img);

/* Butterworth band-pass IIR; coef10 = {b0,b1,b2,a1,a2} x {HP, LP};
 * state4 = per position {w1_hp, w2_hp, w1_lp, w2_lp} */
int   orc_iir_design(float f_low, float f_high, float fs, float *coef10, int *warmup);
void  orc_iir_preseed(const float *coef10, int warmup, const float *x, long n, float *state4);
void  orc_iir_step(const float *coef10, const float *x, long n, float *state4, float *out);

/* adaptive threshold and amplification */
float orc_mag_sum(const float *orig6, long n);
float orc_threshold(const float *orig6, long n, int batch_form);
void  orc_amplify(const float *delta6, const float *orig6, float amp, float thr,
                  int w, int h, float *out6);
float orc_fade_amp(float amp_factor, int frames_before, int warmup);

/* spatial smoothing / luma transfer */
void  orc_box(const float *in, float *out, int w, int h, int r);
void  orc_guided(const float *guide, const float *p, float *out, int w, int h, int r, float eps);
void  orc_gauss5(const float *in, float *out, int w, int h);
void  orc_gray_to_rgb(const float *gray, const float *rgb, int w, int h, int edge_aware, float *out_rgb);

/* window (--haar) temporal filter; ring is [N6][ws] position-major */
void  orc_window_apply(const float *ring, long n, int ws, int head, int bilateral, float *delta);

/* whole-stream drivers (wema_process_frame, wema_batch_process semantics) */
typedef struct {
    int   width, height;
    float fps, amp, f_low, f_high;
    int   window;
    int   edge_aware, bilateral, color, use_iir;
} OrcConfig;

void *orc_stream_new(const OrcConfig *cfg);
void  orc_stream_free(void *s);
int   orc_stream_process(void *s, const float *rgb_in, float *rgb_out);
int   orc_stream_batch(void *s, const float *rgb_in, float *rgb_out, int count);
long  orc_stream_get(void *s, int what, float *dst);
int   orc_stream_frames_processed(void *s);

#endif
