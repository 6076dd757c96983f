// window.cu - the window ("--haar") temporal filter (temporal_filter.c:139-319);
// its deltas are amplified like the IIR's (phase_amp.c:12-56) where the
// inverse DWT stages the coefficients.
//
// The ring holds the last ws frames of every unique coefficient, slot-major
// ([ws][Pu]), so a push is one contiguous plane copy and each thread reads
// its position's history with coalesced loads.  For position u, with the
// window in chronological order x_0..x_{ws-1} (oldest first, centre c = ws/2):
//   delta = x_c - mean(x);
//   bilateral: sigma = max(0.5 * mean|x_t - x_c|, 1e-3),
//              w_t = exp(-(x_t-x_c)^2 / (2 sigma^2)) * exp(-(t-c)^2 / (2 (0.15 ws)^2)),
//              delta = sum w_t (x_t - mean) / sum w_t  (if sum w_t > 1e-8).
// The reference's vectorised reductions and vector expf order these sums
// differently; deltas agree to a few ulp, the bar for this stage.
//
// Precision variant (fp16): the ring's samples are stored as FP16 (rounded to
// nearest on the push) and widened to FP32 as they are read; every sum, the
// mean, the weights and the delta stay FP32.  The ring is the window mode's
// dominant traffic (ws reads per position per frame), so this halves it.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace wema {

constexpr int WIN_THREADS = 256;

__device__ __forceinline__ void put(float* p, float v) { *p = v; }
__device__ __forceinline__ void put(__half* p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ float get(const float* p) { return *p; }
__device__ __forceinline__ float get(const __half* p) { return __half2float(*p); }

template <class T>
__global__ void k_ring_push(const float* coef, int h16, T* ring, long long pu, int slot) {
    T* dst = ring + (long long)slot * pu;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < pu;
         u += (long long)gridDim.x * blockDim.x)
        put(dst + u, pl_ld(coef, u, h16));
}

template <class T>
struct WinDev {
    WindowParams w;
    const T* ring;
    float* delta_out;
};

template <class T>
__global__ void __launch_bounds__(WIN_THREADS) k_window(WinDev<T> a) {
    const long long pu = a.w.pu;
    const int ws = a.w.ws, head = a.w.head, center = ws / 2;
    const float inv_ws = __fdiv_rn(1.0f, (float)ws);
    for (long long u = blockIdx.x * (long long)WIN_THREADS + threadIdx.x; u < pu;
         u += (long long)gridDim.x * WIN_THREADS) {
        float sum = 0.0f, cur = 0.0f;
        for (int t = 0; t < ws; t++) {
            int slot = head + t;
            if (slot >= ws) slot -= ws;
            const float v = get(a.ring + (long long)slot * pu + u);
            sum = __fadd_rn(sum, v);
            if (t == center) cur = v;
        }
        const float mean = __fmul_rn(inv_ws, sum);
        float d = __fadd_rn(cur, -mean);
        if (a.w.bilateral) {
            float mad = 0.0f;
            for (int t = 0; t < ws; t++) {
                int slot = head + t;
                if (slot >= ws) slot -= ws;
                mad = __fadd_rn(mad, fabsf(__fadd_rn(get(a.ring + (long long)slot * pu + u), -cur)));
            }
            const float sigma = fmaxf(__fmul_rn(__fmul_rn(inv_ws, 0.5f), mad), 0.001f);
            const float inv2 = __fdiv_rn(0.5f, __fmul_rn(sigma, sigma));
            float wsum = 0.0f, res = 0.0f;
            for (int t = 0; t < ws; t++) {
                int slot = head + t;
                if (slot >= ws) slot -= ws;
                const float v = get(a.ring + (long long)slot * pu + u);
                const float df = __fadd_rn(v, -cur);
                const float wt = __fmul_rn(expf(-__fmul_rn(__fmul_rn(df, df), inv2)), a.w.time_w[t]);
                wsum = __fadd_rn(wsum, wt);
                res = __fmaf_rn(wt, __fadd_rn(v, -mean), res);
            }
            if (wsum > 1e-8f) d = __fmul_rn(res, __fdiv_rn(1.0f, wsum));
        }
        pl_st(a.delta_out, u, d, a.w.h16);
    }
}

cudaError_t launch_ring_push(const float* coef, int h16, void* ring, int fp16, long long pu, int slot,
                             cudaStream_t st) {
    long long b = (pu + 255) / 256;
    const int g = (int)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
    if (fp16) k_ring_push<__half><<<g, 256, 0, st>>>(coef, h16, static_cast<__half*>(ring), pu, slot);
    else k_ring_push<float><<<g, 256, 0, st>>>(coef, h16, static_cast<float*>(ring), pu, slot);
    return cudaGetLastError();
}

cudaError_t launch_window(const WindowParams& wp, const void* ring, float* delta,
                          cudaStream_t st) {
    long long b = (wp.pu + WIN_THREADS - 1) / WIN_THREADS;
    const int g = (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
    if (wp.fp16) {
        WinDev<__half> a{wp, static_cast<const __half*>(ring), delta};
        k_window<__half><<<g, WIN_THREADS, 0, st>>>(a);
    } else {
        WinDev<float> a{wp, static_cast<const float*>(ring), delta};
        k_window<float><<<g, WIN_THREADS, 0, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace wema
