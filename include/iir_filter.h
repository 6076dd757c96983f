/*
 * iir_filter.h - temporal band-pass filter API of libwema_cuda.
 *
 * Drop-in for the reference's src/iir_filter.h (iir_filter.h:13-134): the
 * same types, field layout and prototypes, so callers that read
 * frames_processed / warmup_frames directly (wema.c:820-832,
 * wema_batch.c:388-411) keep working.  The filter is a cascade of one
 * high-pass (f_low) and one low-pass (f_high) second-order Butterworth
 * section in direct form II transposed, one state pair per section and
 * coefficient position.
 *
 * In this library the per-position state lives in device memory:
 * state_soa points to num_sections {w1, w2} pairs of DEVICE pointers and
 * state is NULL.  Inputs and outputs of the functions below are host arrays.
 */
#ifndef IIR_FILTER_H
#define IIR_FILTER_H

#include <stdbool.h>
#include <stddef.h>

#define IIR_MAX_SECTIONS 4

/* H(z) = (b0 + b1 z^-1 + b2 z^-2) / (1 + a1 z^-1 + a2 z^-2) */
typedef struct {
    float b0, b1, b2;
    float a1, a2;
} BiquadCoeffs;

typedef struct {
    float w1, w2;
} BiquadState;

typedef struct {
    int num_sections;
    BiquadCoeffs sections[IIR_MAX_SECTIONS];
} IIRFilterCoeffs;

typedef struct {
    float *w1;
    float *w2;
} BiquadStateSoA;

typedef struct {
    IIRFilterCoeffs coeffs;
    size_t num_positions;
    BiquadState *state;          /* unused here (NULL) */
    BiquadStateSoA *state_soa;   /* device state, one {w1, w2} per section */
    int warmup_frames;           /* max(30, floor(7 fs / (2 pi f_low))) */
    int frames_processed;
    bool use_simd;               /* true: the AVX-512 path's arithmetic is reproduced */
} IIRTemporalFilter;

/* Butterworth band-pass design (iir_filter.c:70-101).  Returns -1 unless
 * 0 < f_low < f_high < fs/2.  order is clamped to 2..4; two sections
 * (order 2) are what iir_temporal_init uses. */
int iir_design_bandpass(IIRFilterCoeffs *coeffs, float f_low, float f_high, float fs, int order);

/* Allocates device state for num_positions coefficients (iir_filter.c:103-154). */
int iir_temporal_init(IIRTemporalFilter *filt, size_t num_positions,
                      float f_low, float f_high, float fs);
void iir_temporal_free(IIRTemporalFilter *filt);

/* One frame: output[i] = cascade(input[i]) (iir_filter.c:181-264). */
void iir_temporal_process(IIRTemporalFilter *filt, const float *input, float *output);

/* batch_size frames, frame-major [batch][num_positions] (iir_filter.c:266-370). */
void iir_temporal_process_batch(IIRTemporalFilter *filt, const float *input, float *output,
                                int batch_size);

/* frames_processed >= warmup_frames (iir_filter.c:372-374). */
bool iir_temporal_ready(const IIRTemporalFilter *filt);

/* Runs initial_coeffs through the cascade warmup_frames times, once, before
 * the first frame (iir_filter.c:376-471). */
void iir_temporal_preseed(IIRTemporalFilter *filt, const float *initial_coeffs);

#endif /* IIR_FILTER_H */
