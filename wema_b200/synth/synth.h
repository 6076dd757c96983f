/*
 * synth.h - seeded synthetic RGB24 video, the stand-in for the lossless
 * rawvideo/ffv1 inputs of the benchmark workloads.
 *
 * Background: 64 Gaussian blobs (sigma U[8,40] px, uniform centres, signed
 * per-channel amplitudes) on a linear gradient, each channel mapped affinely
 * to [40,210].  Foreground: textured discs (radius 30 px) whose centre moves
 * as c0 + A*sin(2*pi*f*t), sampled bilinearly from a fixed texture with an
 * anti-aliased rim.  Optional global luma flicker.  I.i.d. Gaussian sensor
 * noise, then rounding and clamping to u8.  Every frame is a pure function of
 * (params, frame index), so frames can be produced in any order.
 */
#ifndef WEMA_SYNTH_H
#define WEMA_SYNTH_H

#include <stdint.h>

#define SYNTH_MAX_DISCS 4

typedef struct {
    int      width, height;
    float    fps;
    uint64_t seed;
    int      n_discs;
    float    disc_freq[SYNTH_MAX_DISCS];   /* Hz */
    float    disc_amp[SYNTH_MAX_DISCS];    /* px, peak displacement */
    float    disc_radius;                  /* px */
    float    noise_sigma;                  /* LSB */
    float    flicker_amp;                  /* LSB, 0 = off */
    float    flicker_freq;                 /* Hz */
} SynthParams;

typedef struct SynthStream SynthStream;

SynthStream *synth_new(const SynthParams *p);
void         synth_free(SynthStream *s);
/* Writes frame t as interleaved RGB24 [height][width][3]. */
void         synth_frame(const SynthStream *s, int t, uint8_t *rgb);
/* Writes frames t0 .. t0+count-1 back to back (parallel over frames). */
void         synth_frames(const SynthStream *s, int t0, int count, uint8_t *rgb);

#endif
