/*
 * phase_amp.h - coefficient amplification of libwema_cuda.
 *
 * Drop-in for the reference's src/phase_amp.h (phase_amp.h:18).
 */
#ifndef PHASE_AMP_H
#define PHASE_AMP_H

#include "wema.h"

/* coeffs' six slots = orig + [|orig| > thr] * alpha_l * delta, with
 * thr = 0.2 * mean|orig| evaluated exactly as the reference build does and
 * alpha_0 = alpha / 2 (phase_amp.c:12-56).  delta_coeff and orig_coeff are
 * host arrays of dwt_num_positions(coeffs) floats. */
void coeff_amplify(const float *delta_coeff, const float *orig_coeff, float alpha,
                   DWTCoeffs *coeffs);

#endif /* PHASE_AMP_H */
