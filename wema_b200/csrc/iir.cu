// iir.cu - per-coefficient temporal band-pass (Butterworth HP + LP biquads,
// DF-II transposed), and the adaptive-threshold amplification.
//
// One thread per unique detail coefficient.  The reference filters all six
// slots, but slots 3-5 carry the same input sequence as slots 2-0 and their
// deltas are never read back (dwt.c:749-751), so the unique three suffice.
// State is one float4 per coefficient {w1_hp, w2_hp, w1_lp, w2_lp}.
// Arithmetic is the AVX-512 path's (iir_filter.c:210-224):
//   y = fma(b0, x, w1); w1 = fnma(a1, y, fma(b1, x, w2)); w2 = fnma(a2, y, b2*x)
// except for positions at or past the last full 16-wide block of the 6-slot
// array, which the reference runs in its scalar loop: w2 = fms(b2, x, a2*y)
// (iir_filter.c:231-246).  Amplification (wema.c:726-743):
//   out = |x| > thr ? fma(delta, alpha_l, x) : x,  alpha_0 = alpha/2;
// the per-frame path applies it inside the inverse DWT's staging (dwt.cu), so
// the filter need not wait for the threshold.
//
// Precision variant (fp64): the state and the whole cascade step in double,
// from the FP32-designed coefficients promoted; the band-passed delta is
// rounded to FP32 once.  Poles near the unit circle (a low f_low at a high
// frame rate) accumulate FP32 rounding in the recursive state; this keeps it
// out.  State: {w1_hp, w2_hp} and {w1_lp, w2_lp} as two double2.
#include "cascade.cuh"
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

#include <string.h>

#include <atomic>

namespace wema {

constexpr int IIR_THREADS = 256;
// Positions a thread has in flight (all loads before any use): 2, 4 or 8,
// picked per device by iir_autotune (4 until then).
constexpr int IIR_U = 4;

struct IirDev {
    IirParams p;
    const float* coef;
    long long frame_stride;
    int frames;
    void* state;           // float4 per position, or (fp64) double2[2] per position
    int fp64;
    float* amplified;
    float* delta_out;
    const float* thr;
    const float* amp;      // batch route: per-frame alphas (device)
    float alpha;           // single frame: the channel's alpha
    int warmup;
};

// level of unique position u, and whether its 6-slot index is in the
// reference's scalar tail
__device__ __forceinline__ int level_of(const IirParams& p, long long u, bool& tail) {
    int l = 0;
#pragma unroll
    for (int k = 1; k < 4; k++)
        if (k < p.levels && u >= p.uoff[k]) l = k;
    const long long r = u - p.uoff[l];             // band * n + k, band in 0..2 = slot
    tail = p.off6[l] + r >= p.simd_end;
    return l;
}

__device__ __forceinline__ void iir_preseed_body(const IirDev& a, int block, int nblocks) {
    const long long pu = a.p.uoff[a.p.levels];
    for (long long u = block * (long long)IIR_THREADS + threadIdx.x; u < pu;
         u += (long long)nblocks * IIR_THREADS) {
        const float x = pl_ld(a.coef, u, a.p.h16);
        if (a.fp64) {
            double2* s = static_cast<double2*>(a.state) + 2 * u;
            double2 hp = s[0], lp = s[1];
            for (int it = 0; it < a.warmup; it++) cascade64(a.p.c, hp, lp, x);
            s[0] = hp;
            s[1] = lp;
        } else {
            bool tail;
            level_of(a.p, u, tail);
            float4* s = static_cast<float4*>(a.state) + u;
            float4 st = *s;
            for (int it = 0; it < a.warmup; it++) cascade(a.p.c, st, x, tail);
            *s = st;
        }
    }
}

// A thread takes positions u, u + B, ..., u + (U-1)B (B = the task's threads)
// per pass, so a warp's accesses stay coalesced and U are in flight.
template <int U>
__device__ __forceinline__ void iir_body64(const IirDev& a, int block, int nblocks) {
    const long long pu = a.p.uoff[a.p.levels];
    const long long B = (long long)nblocks * IIR_THREADS;
    const float* __restrict__ coef = a.coef;
    double2* __restrict__ state = static_cast<double2*>(a.state);
    float* __restrict__ dout = a.delta_out;
    for (long long u0 = block * (long long)IIR_THREADS + threadIdx.x; u0 < pu; u0 += U * B) {
        float x[U];
        double2 hp[U], lp[U];
#pragma unroll
        for (int j = 0; j < U; j++) {
            const long long u = u0 + j * B;
            if (u < pu) {
                x[j] = pl_ld(coef, u, a.p.h16);
                hp[j] = __ldcs(state + 2 * u);
                lp[j] = __ldcs(state + 2 * u + 1);
            }
        }
#pragma unroll
        for (int j = 0; j < U; j++) {
            const long long u = u0 + j * B;
            if (u < pu) {
                pl_st(dout, u, cascade64(a.p.c, hp[j], lp[j], x[j]), a.p.h16);
                __stcs(state + 2 * u, hp[j]);
                __stcs(state + 2 * u + 1, lp[j]);
            }
        }
    }
}

// H16: FP16 coefficient / delta planes (planes_fp16), a compile-time constant
template <int U, bool H16>
__device__ __forceinline__ void iir_body_t(const IirDev& a, int block, int nblocks) {
    const long long pu = a.p.uoff[a.p.levels];
    const long long B = (long long)nblocks * IIR_THREADS;
    const float* __restrict__ coef = a.coef;
    float4* __restrict__ state = static_cast<float4*>(a.state);
    float* __restrict__ dout = a.delta_out;
    // a position's 6-slot index is u + uoff[its level] <= u + uoff[last level]:
    // below this bound (and pu) every position exists and none takes the
    // scalar-tail form
    const long long no_tail = min(a.p.simd_end - a.p.uoff[a.p.levels > 0 ? a.p.levels - 1 : 0], pu);
    for (long long u0 = block * (long long)IIR_THREADS + threadIdx.x; u0 < pu; u0 += U * B) {
        float x[U];
        float4 st[U];
#pragma unroll
        for (int j = 0; j < U; j++) {
            const long long u = u0 + j * B;
            if (u < pu) {
                x[j] = pl_ld(coef, u, H16);
                st[j] = __ldcs(state + u);          // touched once per frame: evict first
            }
        }
        if (u0 + (U - 1) * B < no_tail) {           // (uniform but for one grid-stride step)
#pragma unroll
            for (int j = 0; j < U; j++) {
                const long long u = u0 + j * B;
                pl_st(dout, u, cascade(a.p.c, st[j], x[j], false), H16);
                __stcs(state + u, st[j]);
            }
            continue;
        }
#pragma unroll
        for (int j = 0; j < U; j++) {
            const long long u = u0 + j * B;
            if (u < pu) {
                bool tail;
                level_of(a.p, u, tail);
                pl_st(dout, u, cascade(a.p.c, st[j], x[j], tail), H16);
                __stcs(state + u, st[j]);
            }
        }
    }
}

template <int U>
__device__ __forceinline__ void iir_body(const IirDev& a, int block, int nblocks) {
    if (a.fp64) iir_body64<(U > 4 ? 4 : U)>(a, block, nblocks);   // double state: at most 4 in registers
    else if (a.p.h16) iir_body_t<U, true>(a, block, nblocks);
    else iir_body_t<U, false>(a, block, nblocks);
}

__global__ void __launch_bounds__(IIR_THREADS) k_iir_preseed(IirDev a) {
    iir_preseed_body(a, blockIdx.x, gridDim.x);
}
// (U <= 4: 4 CTAs per SM, 64 registers, 32 warps keep the loads in flight;
// U = 8: 2 CTAs per SM, 16 warps with twice the loads each)
template <int U>
__global__ void __launch_bounds__(IIR_THREADS, U <= 4 ? 4 : 2) k_iir(IirDev a) {
    iir_body<U>(a, blockIdx.x, gridDim.x);
}
// batched: task = one (stream, channel); the task's grid x is its block count
template <int U>
__global__ void __launch_bounds__(IIR_THREADS, U <= 4 ? 4 : 2)
    k_iir_multi(const IirDev* __restrict__ as, const int* __restrict__ map, int preseed) {
    const TaskBlock t = task_block(map, blockIdx.x);
    const int nb = map[map[0] + 2 + t.task];
    if (preseed) iir_preseed_body(as[t.task], t.x, nb);
    else iir_body<U>(as[t.task], t.x, nb);
}

// ---- positions per thread, per device
static std::atomic<int> g_positions[64];

static int device_now() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

int iir_positions(int dev) {
    const int u = (dev >= 0 && dev < 64) ? g_positions[dev].load() : 0;
    return u ? u : IIR_U;
}

bool iir_set_positions(int dev, int u) {
    if (dev < 0 || dev >= 64 || (u != 2 && u != 4 && u != 8)) return false;
    g_positions[dev].store(u);
    return true;
}

template <int U>
static void launch_k_iir(int blocks, const IirDev& a, cudaStream_t st) {
    k_iir<U><<<blocks, IIR_THREADS, 0, st>>>(a);
}

__global__ void __launch_bounds__(IIR_THREADS) k_amplify(IirDev a) {
    const long long pu = a.p.uoff[a.p.levels];
    const float thr = *a.thr;
    const float alpha0 = __fmul_rn(a.alpha, 0.5f);
    for (long long u = blockIdx.x * (long long)IIR_THREADS + threadIdx.x; u < pu;
         u += (long long)gridDim.x * IIR_THREADS) {
        bool tail;
        const int l = level_of(a.p, u, tail);
        const float x = pl_ld(a.coef, u, a.p.h16);
        a.amplified[u] = fabsf(x) > thr ? __fmaf_rn(pl_ld(a.delta_out, u, a.p.h16), l == 0 ? alpha0 : a.alpha, x) : x;
    }
}

static int grid_for_u(long long n, int u) {
    long long b = (n + (long long)IIR_THREADS * u - 1) / ((long long)IIR_THREADS * u);
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}
static int grid_for(long long n) { return grid_for_u(n, iir_positions(device_now())); }

cudaError_t launch_iir_preseed(const IirParams& p, const float* coef, void* state, int fp64, int warmup,
                               cudaStream_t st) {
    IirDev a{};
    a.p = p;
    a.coef = coef;
    a.state = state;
    a.fp64 = fp64;
    a.warmup = warmup;
    k_iir_preseed<<<grid_for(p.uoff[p.levels]), IIR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_iir(const IirParams& p, const float* coef, void* state, int fp64, float* delta,
                       cudaStream_t st) {
    IirDev a{};
    a.p = p;
    a.coef = coef;
    a.state = state;
    a.fp64 = fp64;
    a.delta_out = delta;
    const int u = iir_positions(device_now());
    const int g = grid_for_u(p.uoff[p.levels], u);
    if (u == 2) launch_k_iir<2>(g, a, st);
    else if (u == 8) launch_k_iir<8>(g, a, st);
    else launch_k_iir<4>(g, a, st);
    return cudaGetLastError();
}

cudaError_t launch_amplify(const IirParams& p, const float* coef, const float* delta,
                           const float* thr, float alpha, float* amplified, cudaStream_t st) {
    IirDev a{};
    a.p = p;
    a.coef = coef;
    a.delta_out = const_cast<float*>(delta);
    a.thr = thr;
    a.alpha = alpha;
    a.amplified = amplified;
    k_amplify<<<grid_for(p.uoff[p.levels]), IIR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

// ---- batched filter (the host fills one IirDev per stream and channel)
size_t iir_args_bytes() { return sizeof(IirDev); }

unsigned iir_args_fill(void* dst, const IirParams& p, const float* coef, void* state, int fp64, float* delta,
                       int warmup) {
    IirDev a{};
    a.p = p;
    a.coef = coef;
    a.state = state;
    a.fp64 = fp64;
    a.delta_out = delta;
    a.warmup = warmup;
    memcpy(dst, &a, sizeof a);
    return (unsigned)grid_for(p.uoff[p.levels]);
}

cudaError_t launch_iir_multi(const void* d_args, const int* d_map, unsigned blocks, int preseed,
                             cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    const IirDev* as = static_cast<const IirDev*>(d_args);
    const int u = iir_positions(device_now());
    if (u == 2) k_iir_multi<2><<<blocks, IIR_THREADS, 0, st>>>(as, d_map, preseed);
    else if (u == 8) k_iir_multi<8><<<blocks, IIR_THREADS, 0, st>>>(as, d_map, preseed);
    else k_iir_multi<4><<<blocks, IIR_THREADS, 0, st>>>(as, d_map, preseed);
    return cudaGetLastError();
}

// ---- the autotuner: times the filter step at 2, 4 and 8 positions per thread
// on a synthetic 2^23-position plane (a 3840x2160 frame's detail count) and
// keeps the fastest for this device - the default 4 unless another is faster
// by more than 3% (the trial runs alone; in a tick the filter shares the GPU
// with the threshold, so small margins are not worth a change).  The
// arithmetic per position does not depend on the choice, so results are
// bit-identical whatever it picks.
cudaError_t iir_autotune(int dev, float ms[3], int* chosen) {
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    const long long n = 1LL << 23;
    float *coef = nullptr, *delta = nullptr;
    float4* state = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    auto done = [&](cudaError_t r) {
        if (coef) cudaFree(coef);
        if (delta) cudaFree(delta);
        if (state) cudaFree(state);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
        return r;
    };
    if ((e = cudaMalloc(&coef, n * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&delta, n * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&state, n * sizeof(float4))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(coef, 0, n * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(state, 0, n * sizeof(float4))) != cudaSuccess) return done(e);
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return done(e);
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) return done(e);
    IirDev a{};
    a.p.levels = 1;
    a.p.uoff[1] = n;
    a.p.n[0] = n / 3;
    a.p.off6[1] = 2 * n;
    a.p.simd_end = (2 * n) & ~15LL;
    a.coef = coef;
    a.state = state;
    a.delta_out = delta;
    const int us[3] = {2, 4, 8};
    for (int k = 0; k < 3; k++) {
        const int u = us[k], g = grid_for_u(n, u);
        for (int rep = 0; rep < 6; rep++) {          // one warm-up, five timed
            if (rep == 1 && (e = cudaEventRecord(e0, st)) != cudaSuccess) return done(e);
            if (u == 2) launch_k_iir<2>(g, a, st);
            else if (u == 8) launch_k_iir<8>(g, a, st);
            else launch_k_iir<4>(g, a, st);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return done(e);
        if ((e = cudaEventRecord(e1, st)) != cudaSuccess) return done(e);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return done(e);
        float t = 0.f;
        if ((e = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) return done(e);
        ms[k] = t / 5.f;
    }
    int best = IIR_U;
    float best_ms = ms[1];
    for (int k = 0; k < 3; k++)
        if (ms[k] < 0.97f * best_ms) {
            best = us[k];
            best_ms = ms[k];
        }
    iir_set_positions(dev, best);
    *chosen = best;
    return done(cudaSuccess);
}

}  // namespace wema
