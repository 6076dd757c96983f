/*
 * temporal_filter.h - window ("--haar") temporal filter API of libwema_cuda.
 *
 * Drop-in for the reference's src/temporal_filter.h (temporal_filter.h:18-66).
 * The history ring is device memory (TemporalBuffer.phase_buffer); the
 * newest coefficients (amplitude) and the output deltas are host arrays.
 */
#ifndef TEMPORAL_FILTER_H
#define TEMPORAL_FILTER_H

#include "wema.h"

/* Records the normalised band and the window's level count; the band does not
 * change the output (the reference's per-scale selection is commented out,
 * temporal_filter.c:253-269). */
int  temporal_filter_init(TemporalFilter *filt, float f_low, float f_high, int window_size);
void temporal_filter_free(TemporalFilter *filt);

int  temporal_buffer_init(TemporalBuffer *buf, const DWTCoeffs *coeffs, int window_size);
void temporal_buffer_free(TemporalBuffer *buf);

/* Appends the frame's six-slot coefficients (temporal_filter.c:139-168). */
void temporal_buffer_push(TemporalBuffer *buf, const DWTCoeffs *coeffs);

/* delta = centre sample - window mean, optionally bilateral-weighted
 * (temporal_filter.c:170-319); zeros until the window is full. */
void temporal_filter_apply(const TemporalFilter *filt, const TemporalBuffer *buf,
                           float *delta_phi_filtered, bool bilateral);

static inline bool temporal_buffer_ready(const TemporalBuffer *buf) {
    return buf->filled >= buf->window_size;
}

int temporal_buffer_output_count(const TemporalBuffer *buf);

#endif /* TEMPORAL_FILTER_H */
