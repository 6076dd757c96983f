/*
 * wema.h - core types and the per-frame pipeline API of libwema_cuda.
 *
 * Drop-in for the reference's src/wema.h (wema.h:19-283): identical constants,
 * type names, field layouts and prototypes, so the reference's C11 callers
 * (main.c:220-496) link against libwema_cuda unchanged.  The work runs on the
 * GPU; Frame data and DWTCoeffs subband arrays stay host memory with the
 * reference's meaning, and the per-stream temporal state stays in device
 * memory between calls.  Internal work buffers of WemaContext that the
 * reference fills as by-products (gray_in, delta_phi, prev_coeffs, ...) are
 * not mirrored to the host; wema_cuda.h has the inspection calls.
 */
#ifndef WEMA_H
#define WEMA_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#include "iir_filter.h"

#define WEMA_MAX_LEVELS          4
#define WEMA_NUM_ORIENTATIONS    6    /* 3 unique detail bands + 3 mirrored slots */
#define WEMA_TEMPORAL_WINDOW_DEF 32
#define WEMA_TEMPORAL_WINDOW_MAX 256

typedef struct {
    float *data;      /* [height][width][channels], values in [0,1] */
    int    width;
    int    height;
    int    channels;
} Frame;

typedef struct {
    float *coeffs;    /* [height][width] */
    int    width;
    int    height;
} Subband;

/* Slots per level: 0 LH, 1 HH, 2 HL, 3 HL, 4 HH, 5 LH (dwt.c:679-687). */
typedef struct {
    float  *lowpass;
    int     lowpass_w;
    int     lowpass_h;
    Subband subbands[WEMA_MAX_LEVELS][WEMA_NUM_ORIENTATIONS];
    int     num_levels;
    int     orig_width;
    int     orig_height;
} DWTCoeffs;

/* Window ("--haar") mode history.  In this library phase_buffer is a DEVICE
 * ring of window_size frames; amplitude (the newest coefficients) is host. */
typedef struct {
    float  *phase_buffer;
    float  *amplitude;
    float  *dc_phase;
    size_t  num_positions;
    int     window_size;
    int     head;
    int     filled;
    int     num_levels;
    int     widths[WEMA_MAX_LEVELS];
    int     heights[WEMA_MAX_LEVELS];
} TemporalBuffer;

typedef struct {
    float *lp_filter;
    float *hp_filter;
    int    filter_len;
    float  f_low_norm;
    float  f_high_norm;
    int    temporal_levels;
} TemporalFilter;

typedef struct {
    int    width;
    int    height;
    float  fps;

    float  amp_factor;
    float  f_low;
    float  f_high;
    int    num_levels;
    int    temporal_window;
    bool   edge_aware;
    bool   bilateral_temp;
    bool   color_mode;
    bool   use_iir;

    float  f_low_norm;
    float  f_high_norm;

    DWTCoeffs      *coeffs;
    TemporalBuffer *temporal_buf;
    TemporalFilter *temporal_filt;

    DWTCoeffs      *coeffs_cb;
    DWTCoeffs      *coeffs_cr;
    TemporalBuffer *temporal_buf_cb;
    TemporalBuffer *temporal_buf_cr;

    IIRTemporalFilter *iir_filt;
    IIRTemporalFilter *iir_filt_cb;
    IIRTemporalFilter *iir_filt_cr;
    float             *prev_coeffs;
    float             *prev_coeffs_cb;
    float             *prev_coeffs_cr;

    float  *gray_in;
    float  *gray_out;
    float  *delta_phi;

    float  *cb_in;
    float  *cr_in;
    float  *cb_out;
    float  *cr_out;
    float  *delta_cb;
    float  *delta_cr;

    float  *delta_buf;
    float  *smooth_buf;
    float  *guide_buf;
    float  *guided_work[4];
} WemaContext;

typedef struct {
    int     in_pid;
    int     in_fd;
    int     out_pid;
    int     out_fd;
    int     width;
    int     height;
    float   fps;
    int64_t total_frames;
    char   *input_path;
    uint8_t *raw_buffer;
    size_t   buffer_size;
} FFmpegIO;

typedef struct {
    char   *input_path;
    char   *output_path;
    float   amp_factor;
    float   f_low;
    float   f_high;
    int     temporal_window;
    char   *ff_codec;
    char   *ff_options;
    bool    verbose;
    bool    edge_aware;
    bool    bilateral_temp;
    bool    color_mode;
    bool    use_iir;
    int     batch_size;
    int     num_threads;
} WemaConfig;

#define WEMA_BATCH_SIZE_DEF 64
#define WEMA_BATCH_SIZE_MAX 256

typedef struct {
    int     batch_size;
    int     num_threads;
    size_t  num_positions;
    int     width;
    int     height;
    float  *coeffs_batch;
    float  *delta_batch;
    float  *gray_batch;
    float  *out_batch;
    DWTCoeffs *dwt_batch;
    float  *smooth_buffers;
    int     smooth_buf_stride;
    int     frames_in_batch;
    int     warmup_frames;
} WemaBatchContext;

/* --- pipeline (wema.c:359-960) ------------------------------------------ */
int  wema_init(WemaContext *ctx, int width, int height, float fps,
               float amp_factor, float f_low, float f_high,
               int temporal_window);
int  wema_init_color(WemaContext *ctx);
int  wema_init_iir(WemaContext *ctx);
int  wema_init_iir_color(WemaContext *ctx);
void wema_free(WemaContext *ctx);
/* One frame of float RGB in [0,1], host memory; mirrors wema_process_frame
 * (wema.c:746-952) including the window-mode pass-through while filling. */
int  wema_process_frame(WemaContext *ctx, const Frame *in, Frame *out);
int  wema_flush(WemaContext *ctx, Frame *out);   /* always -1, as the reference */
bool wema_ready(const WemaContext *ctx);

/* --- batch route (wema_batch.c:138-457) --------------------------------- */
int  wema_batch_init(WemaBatchContext *batch, const WemaContext *wema,
                     int batch_size, int num_threads);
void wema_batch_free(WemaBatchContext *batch);
int  wema_batch_process(WemaContext *wema, WemaBatchContext *batch,
                        const Frame *frames_in, Frame *frames_out,
                        int frame_count);

/* --- frame utilities (wema.c:29-353) ------------------------------------ */
int  frame_alloc(Frame *frame, int width, int height, int channels);
void frame_free(Frame *frame);
void frame_rgb_to_gray(const Frame *rgb, float *gray);
void frame_gray_to_rgb(const float *gray, const Frame *orig, Frame *out,
                       float *delta_buf, float *smooth_buf);

#endif /* WEMA_H */
