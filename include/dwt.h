/*
 * dwt.h - 2D CDF 9/7 lifting DWT of libwema_cuda.
 *
 * Drop-in for the reference's src/dwt.h (dwt.h:15-45).  DWTCoeffs keeps host
 * subband arrays in the reference's six-slot layout; the transforms run on the
 * GPU (host -> device copy, kernels, device -> host copy).
 */
#ifndef DWT_H
#define DWT_H

#include "wema.h"

/* Allocates zeroed host subbands of (w+1)/2 x (h+1)/2 per level
 * (dwt.c:598-632).  Returns 0 or -1. */
int dwt_init(DWTCoeffs *coeffs, int width, int height, int num_levels);

void dwt_free(DWTCoeffs *coeffs);

/* Forward transform of a [height][width] image into coeffs (dwt.c:645-703).
 * Subband entries not covered by an odd-sized level keep the previous
 * level's value at the same index (0 at level 0). */
void dwt_forward(const float *image, int width, int height, DWTCoeffs *coeffs);

/* Inverse transform from slots 0-2 and the lowpass (dwt.c:705-767). */
void dwt_inverse(const DWTCoeffs *coeffs, float *image);

size_t dwt_num_positions(const DWTCoeffs *coeffs);

/* Halve the smaller side while it is >= 16, at most 4 times, at least 1
 * level (dwt.c:588-596). */
int dwt_compute_levels(int width, int height);

#endif /* DWT_H */
