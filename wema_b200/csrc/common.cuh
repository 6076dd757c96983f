// common.cuh - shared definitions for the sm_100a kernels and the host runtime.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#define WEMA_MAX_LEV 4

namespace wema {

// CDF 9/7 lifting constants of the reference (dwt.c:31-36), as float.
constexpr float kAlpha = -1.586134342059924f;
constexpr float kBeta = -0.052980118572961f;
constexpr float kGamma = 0.882911075530934f;
constexpr float kDelta = 0.443506852043971f;
constexpr float kK = 1.149604398860241f;
constexpr float kKInv = 1.0f / 1.149604398860241f;

// Geometry of one frame's 2D pyramid.  Level l (0-based) transforms an
// input of in_w[l] x in_h[l] samples into four (in_w+1)/2 x (in_h+1)/2
// subbands (dwt.c:598-632); the coarsest LL is the lowpass.
//
// Device storage keeps the three unique detail bands of each level, band
// order LH, HH, HL (the reference's slots 0, 1, 2; slots 3-5 mirror 2, 1, 0):
//   coef[ uoff[l] + band * n[l] + y * sw[l] + x ]
// The reference's 6-slot flat index of (l, slot, k) is off6[l] + slot*n[l] + k.
struct Geom {
    int w, h, levels;
    int in_w[WEMA_MAX_LEV + 1], in_h[WEMA_MAX_LEV + 1];   // in_w[levels] = lowpass
    int sw[WEMA_MAX_LEV], sh[WEMA_MAX_LEV];
    long long n[WEMA_MAX_LEV];        // sw*sh
    long long uoff[WEMA_MAX_LEV + 1]; // unique-plane offsets; uoff[levels] = Pu
    long long off6[WEMA_MAX_LEV + 1]; // 6-slot offsets; off6[levels] = N6
    long long pixels;
    long long low_n;                  // lowpass samples
};

inline int compute_levels(int w, int h) {   // dwt.c:588-596
    int m = w < h ? w : h, l = 0;
    while (m >= 16 && l < WEMA_MAX_LEV) { m /= 2; l++; }
    return l > 0 ? l : 1;
}

inline Geom make_geom(int w, int h, int levels = -1) {
    Geom g{};
    g.w = w;
    g.h = h;
    g.levels = levels > 0 ? levels : compute_levels(w, h);
    g.in_w[0] = w;
    g.in_h[0] = h;
    long long u = 0, s6 = 0;
    for (int l = 0; l < g.levels; l++) {
        g.sw[l] = (g.in_w[l] + 1) / 2;
        g.sh[l] = (g.in_h[l] + 1) / 2;
        g.in_w[l + 1] = g.sw[l];
        g.in_h[l + 1] = g.sh[l];
        g.n[l] = (long long)g.sw[l] * g.sh[l];
        g.uoff[l] = u;
        g.off6[l] = s6;
        u += 3 * g.n[l];
        s6 += 6 * g.n[l];
    }
    g.uoff[g.levels] = u;
    g.off6[g.levels] = s6;
    g.pixels = (long long)w * h;
    g.low_n = (long long)g.in_w[g.levels] * g.in_h[g.levels];
    return g;
}

// Number of leading elements of an n-element loop that the reference's
// GCC-vectorised code handles with vector instructions (an 8-wide body, then
// at most one 4-wide block); the scalar epilogue evaluates some expressions
// in a different order.
__host__ __device__ inline long long vec_cover(long long n) {
    long long main = (n - 1 <= 6) ? 0 : (n & ~7LL);
    long long rem = n - main;
    return main + (rem >= 4 ? 4 : 0);
}

// Luma as the reference build evaluates 0.299R+0.587G+0.114B (wema.c:42-51):
// vector body and scalar tail differ in FMA order.
__device__ __forceinline__ float luma_vec(float r, float g, float b) {
    return __fmaf_rn(b, 0.114f, __fmaf_rn(r, 0.299f, __fmul_rn(g, 0.587f)));
}
__device__ __forceinline__ float luma_tail(float r, float g, float b) {
    return __fmaf_rn(r, 0.299f, __fmaf_rn(g, 0.587f, __fmul_rn(b, 0.114f)));
}

// RGB -> YCbCr (wema.c:60-78), vector-body and tail forms.
__device__ __forceinline__ void ycbcr_vec(float r, float g, float b, float& y, float& cb, float& cr) {
    y = luma_vec(r, g, b);
    cb = __fadd_rn(__fmaf_rn(-g, 0.331f, 0.5f), __fmaf_rn(r, -0.169f, __fmul_rn(b, 0.5f)));
    cr = __fmaf_rn(-b, 0.081f, __fmaf_rn(-g, 0.419f, __fmul_rn(__fadd_rn(r, 1.0f), 0.5f)));
}
__device__ __forceinline__ void ycbcr_tail(float r, float g, float b, float& y, float& cb, float& cr) {
    y = luma_tail(r, g, b);
    cb = __fadd_rn(__fmaf_rn(-g, 0.331f, __fmul_rn(b, 0.5f)), __fmaf_rn(r, -0.169f, 0.5f));
    cr = __fmaf_rn(__fadd_rn(r, 1.0f), 0.5f, -__fmaf_rn(g, 0.419f, __fmul_rn(b, 0.081f)));
}

// Pyramid planes are FP32, or FP16 in the planes_fp16 precision variant
// (arithmetic stays FP32): an element of plane p at index i, with the
// storage type given by h (uniform over a launch).  Host-side pointers to
// FP16 planes keep the float* type; plane_at() offsets them by elements.
__device__ __forceinline__ float pl_ld(const float* p, long long i, bool h) {
    return h ? __half2float(__ldg(reinterpret_cast<const __half*>(p) + i)) : __ldg(p + i);
}
__device__ __forceinline__ void pl_st(float* p, long long i, float v, bool h) {
    if (h) reinterpret_cast<__half*>(p)[i] = __float2half_rn(v);
    else p[i] = v;
}
__host__ __device__ inline float* plane_at(float* p, long long i, bool h) {
    return p ? (h ? reinterpret_cast<float*>(reinterpret_cast<__half*>(p) + i) : p + i) : nullptr;
}
__host__ __device__ inline const float* plane_at(const float* p, long long i, bool h) {
    return p ? (h ? reinterpret_cast<const float*>(reinterpret_cast<const __half*>(p) + i) : p + i) : nullptr;
}

__device__ __forceinline__ float clamp01(float v) {
    v = v < 1.0f ? v : 1.0f;
    return v > 0.0f ? v : 0.0f;
}

// u8 -> float: fl(i / 255), as the reference's frame reader converts
// (ffmpeg_io.c:293).  With x = i / 256 (exact), fma(x, fl(1/255), x) =
// x * (1 + fl(1/255)) rounded once equals the correctly rounded i / 255 for
// every i in 0..255 (checked exhaustively in tests/test_u8_exact.py).  x is
// made without a conversion instruction (those share the narrow XU pipe):
// the float with bits 0x47000000 | i is 32768 + i/256 exactly (exponent 15,
// mantissa step 2^-8), and subtracting 32768 is exact.
__device__ __forceinline__ float byte_of(uint32_t w, int k) {   // byte k of w
    const float x = __fsub_rn(__uint_as_float(__byte_perm(w, 0x47000000u, 0x7540u | (unsigned)k)), 32768.0f);
    return __fmaf_rn(x, 1.0f / 255.0f, x);
}
__device__ __forceinline__ float u8f(uint32_t i) { return byte_of(i, 0); }

// float in [0,1] -> u8 the way the reference's frame writer quantises
// (ffmpeg_io.c:305-310): v*255, +0.5, truncate; each op rounded alone.  The
// truncation without a conversion instruction: y = v*255 + 0.5 lies in
// [0.5, 255.5], so y + 2^23 rounded down is 2^23 + floor(y), whose low
// mantissa byte is the result.
__device__ __forceinline__ uint32_t quant_bits(float v) {
    const float y = __fadd_rn(__fmul_rn(v, 255.0f), 0.5f);
    return __float_as_uint(__fadd_rd(y, 8388608.0f));
}
// the same after the clamp to [0, 1]
__device__ __forceinline__ uint8_t quant_u8(float v) { return (uint8_t)(quant_bits(clamp01(v)) & 0xffu); }

// YCbCr -> RGB with clamp (wema.c:80-102)
__device__ __forceinline__ void ycbcr_to_rgb(float y, float cb, float cr, float& r, float& g, float& b) {
    float cbv = __fadd_rn(cb, -0.5f), crv = __fadd_rn(cr, -0.5f);
    r = clamp01(__fmaf_rn(crv, 1.402f, y));
    g = clamp01(__fadd_rn(y, -__fmaf_rn(cbv, 0.344f, __fmul_rn(crv, 0.714f))));
    b = clamp01(__fmaf_rn(cbv, 1.772f, y));
}

}  // namespace wema
