// cascade.cuh - one step of the temporal band-pass (Butterworth high-pass then
// low-pass biquad, DF-II transposed) for one coefficient, shared by the
// filter kernels (iir.cu) and the forward transform, which runs the step on
// each coefficient as it writes it (dwt.cu).
//
// Arithmetic of the reference's AVX-512 path (iir_filter.c:210-224):
//   y = fma(b0, x, w1); w1 = fnma(a1, y, fma(b1, x, w2)); w2 = fnma(a2, y, b2*x)
// except for positions at or past the last full 16-wide block of the 6-slot
// array, which the reference runs in its scalar loop: w2 = fms(b2, x, a2*y)
// (iir_filter.c:231-246).  c = {b0,b1,b2,a1,a2} high-pass, then low-pass.
#pragma once

#include "common.cuh"

namespace wema {

__device__ __forceinline__ float cascade(const float* c, float4& st, float x, bool tail) {
    // high-pass section
    float y = __fmaf_rn(c[0], x, st.x);
    float w1 = __fmaf_rn(-c[3], y, __fmaf_rn(c[1], x, st.y));
    float w2 = tail ? __fmaf_rn(c[2], x, -__fmul_rn(c[4], y)) : __fmaf_rn(-c[4], y, __fmul_rn(c[2], x));
    st.x = w1;
    st.y = w2;
    x = y;
    // low-pass section
    y = __fmaf_rn(c[5], x, st.z);
    w1 = __fmaf_rn(-c[8], y, __fmaf_rn(c[6], x, st.w));
    w2 = tail ? __fmaf_rn(c[7], x, -__fmul_rn(c[9], y)) : __fmaf_rn(-c[9], y, __fmul_rn(c[7], x));
    st.z = w1;
    st.w = w2;
    return y;
}

// the fp64 variant of cascade(): one rounding, at the end
__device__ __forceinline__ float cascade64(const float* c, double2& hp, double2& lp, float xf) {
    const double x = (double)xf;
    double y = fma((double)c[0], x, hp.x);
    hp.x = fma(-(double)c[3], y, fma((double)c[1], x, hp.y));
    hp.y = fma(-(double)c[4], y, (double)c[2] * x);
    const double x2 = y;
    y = fma((double)c[5], x2, lp.x);
    lp.x = fma(-(double)c[8], y, fma((double)c[6], x2, lp.y));
    lp.y = fma(-(double)c[9], y, (double)c[7] * x2);
    return __double2float_rn(y);
}

}  // namespace wema
