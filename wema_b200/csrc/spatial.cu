// spatial.cu - luma-delta smoothing and transfer to RGB, fused with the u8
// output (wema.c:289-335, wema_batch.c:311-346).
//
// guide I = luma of the input frame (same evaluation as the DWT input),
// p = gray_out - I, smoothed by the guided filter (radius 4, eps 0.01,
// wema.c:173-230) or, with edge-aware off, the 5-tap [1 4 6 4 1]/16 blur
// with border renormalisation (wema.c:236-283); then
// out = clamp01(RGB + smooth) and u8 = (uint8)(v*255 + 0.5).
//
// One CTA produces a TS x TS output tile.  The guided filter's two rounds of
// radius-4 box means need an 8-pixel halo; every box mean is the clipped
// window's sum divided by the clipped count, rows first then columns (the
// reference's definition), computed here by direct 9-term sums in shared
// memory rather than by the reference's FP32 running prefix sums - the two
// differ in the last bits only, which the u8 output absorbs (<= 1 LSB).
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

namespace wema {

constexpr int TS = 32;
constexpr int GR = 4;                   // guided-filter radius
constexpr int H0 = 2 * GR;              // input halo
constexpr int R0 = TS + 2 * H0;         // 48: I, p region
constexpr int R1 = TS + 2 * GR;         // 40: first-round means, a, b
constexpr int SP_THREADS = 256;

struct SpArgs { TransferParams p; };

__device__ __forceinline__ void load_rgb(const TransferParams& p, const float* lut, long long pi,
                                         float& r, float& g, float& b) {
    if (p.src_u8) {
        const uint8_t* q = p.src_u8 + 3 * pi;
        r = lut[q[0]]; g = lut[q[1]]; b = lut[q[2]];
    } else {
        const float* q = p.src_f32 + 3 * pi;
        r = q[0]; g = q[1]; b = q[2];
    }
}

__device__ __forceinline__ void store_rgb(const TransferParams& p, long long pi, float r, float g,
                                          float b, float dy) {
    r = clamp01(__fadd_rn(r, dy));
    g = clamp01(__fadd_rn(g, dy));
    b = clamp01(__fadd_rn(b, dy));
    if (p.out_u8) {
        uint8_t* d = p.out_u8 + 3 * pi;
        d[0] = quant_u8(r); d[1] = quant_u8(g); d[2] = quant_u8(b);
    }
    if (p.out_f32) {
        float* d = p.out_f32 + 3 * pi;
        d[0] = r; d[1] = g; d[2] = b;
    }
}

struct GuidedSmem {
    float I[R0][R0 + 1];
    float P[R0][R0 + 1];
    float hm[4][R0][R1 + 1];     // row means of I, p, I*I, I*p over the region rows
    float A[R1][R1 + 1];
    float B[R1][R1 + 1];
    float ha[2][R1][TS + 1];     // row means of a, b
};

__device__ __forceinline__ void guided_body(const TransferParams& p, int bx, int by) {
    extern __shared__ unsigned char raw[];
    GuidedSmem& S = *reinterpret_cast<GuidedSmem*>(raw);
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += SP_THREADS) lut[i] = __fdiv_rn((float)i, 255.0f);
    const int W = p.w, H = p.h;
    const int x0 = bx * TS, y0 = by * TS;
    const int gx0 = x0 - H0, gy0 = y0 - H0;      // region origin (may be negative)
    __syncthreads();

    // I and p over the 48x48 region (positions outside the image unused)
    for (int k = threadIdx.x; k < R0 * R0; k += SP_THREADS) {
        const int ly = k / R0, lx = k % R0;
        const int gx = gx0 + lx, gy = gy0 + ly;
        float I = 0.f, P = 0.f;
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            const long long pi = (long long)gy * W + gx;
            float r, g, b;
            load_rgb(p, lut, pi, r, g, b);
            I = pi < p.vec_end ? luma_vec(r, g, b) : luma_tail(r, g, b);
            P = __fadd_rn(p.gray_out[pi], -I);
        }
        S.I[ly][lx] = I;
        S.P[ly][lx] = P;
    }
    __syncthreads();

    // row means for columns of the 40-wide first-round region
    for (int k = threadIdx.x; k < R0 * R1; k += SP_THREADS) {
        const int ly = k / R1, cx = k % R1;
        const int gx = x0 - GR + cx;
        const int gy = gy0 + ly;
        if (gx < 0 || gx >= W || gy < 0 || gy >= H) continue;
        const int a = max(gx - GR, 0), b = min(gx + GR + 1, W);
        float sI = 0.f, sP = 0.f, sII = 0.f, sIP = 0.f;
        for (int x = a; x < b; x++) {
            const float I = S.I[ly][x - gx0], P = S.P[ly][x - gx0];
            sI = __fadd_rn(sI, I);
            sP = __fadd_rn(sP, P);
            sII = __fadd_rn(sII, __fmul_rn(I, I));
            sIP = __fadd_rn(sIP, __fmul_rn(I, P));
        }
        const float cnt = (float)(b - a);
        S.hm[0][ly][cx] = __fdiv_rn(sI, cnt);
        S.hm[1][ly][cx] = __fdiv_rn(sP, cnt);
        S.hm[2][ly][cx] = __fdiv_rn(sII, cnt);
        S.hm[3][ly][cx] = __fdiv_rn(sIP, cnt);
    }
    __syncthreads();

    // column means -> a, b over the 40x40 first-round region
    for (int k = threadIdx.x; k < R1 * R1; k += SP_THREADS) {
        const int cy = k / R1, cx = k % R1;
        const int gx = x0 - GR + cx, gy = y0 - GR + cy;
        if (gx < 0 || gx >= W || gy < 0 || gy >= H) continue;
        const int a = max(gy - GR, 0), b = min(gy + GR + 1, H);
        float m[4] = {0.f, 0.f, 0.f, 0.f};
        for (int y = a; y < b; y++)
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fadd_rn(m[q], S.hm[q][y - gy0][cx]);
        const float cnt = (float)(b - a);
#pragma unroll
        for (int q = 0; q < 4; q++) m[q] = __fdiv_rn(m[q], cnt);
        const float mI = m[0], mP = m[1], cII = m[2], cIP = m[3];
        const float av = __fdiv_rn(__fmaf_rn(-mI, mP, cIP), __fmaf_rn(-mI, mI, __fadd_rn(cII, 0.01f)));
        S.A[cy][cx] = av;
        S.B[cy][cx] = __fmaf_rn(-av, mI, mP);
    }
    __syncthreads();

    // second round: row means of a, b for the tile's columns
    for (int k = threadIdx.x; k < R1 * TS; k += SP_THREADS) {
        const int cy = k / TS, tx = k % TS;
        const int gx = x0 + tx, gy = y0 - GR + cy;
        if (gx >= W || gy < 0 || gy >= H) continue;
        const int a = max(gx - GR, 0), b = min(gx + GR + 1, W);
        float sa = 0.f, sb = 0.f;
        for (int x = a; x < b; x++) {
            sa = __fadd_rn(sa, S.A[cy][x - (x0 - GR)]);
            sb = __fadd_rn(sb, S.B[cy][x - (x0 - GR)]);
        }
        const float cnt = (float)(b - a);
        S.ha[0][cy][tx] = __fdiv_rn(sa, cnt);
        S.ha[1][cy][tx] = __fdiv_rn(sb, cnt);
    }
    __syncthreads();

    for (int k = threadIdx.x; k < TS * TS; k += SP_THREADS) {
        const int ty = k / TS, tx = k % TS;
        const int gx = x0 + tx, gy = y0 + ty;
        if (gx >= W || gy >= H) continue;
        const int a = max(gy - GR, 0), b = min(gy + GR + 1, H);
        float sa = 0.f, sb = 0.f;
        for (int y = a; y < b; y++) {
            sa = __fadd_rn(sa, S.ha[0][y - (y0 - GR)][tx]);
            sb = __fadd_rn(sb, S.ha[1][y - (y0 - GR)][tx]);
        }
        const float cnt = (float)(b - a);
        const float ma = __fdiv_rn(sa, cnt), mb = __fdiv_rn(sb, cnt);
        const float I = S.I[gy - gy0][gx - gx0];
        const float dy = __fmaf_rn(ma, I, mb);
        const long long pi = (long long)gy * W + gx;
        float r, g, bb;
        load_rgb(p, lut, pi, r, g, bb);
        store_rgb(p, pi, r, g, bb, dy);
    }
}

// 5-tap Gaussian fallback: halo 2
constexpr int GH = 2;
constexpr int RG = TS + 2 * GH;

__device__ __forceinline__ void gauss_body(const TransferParams& p, int bx, int by) {
    __shared__ float P[RG][RG + 1];
    __shared__ float T[RG][TS + 1];
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += SP_THREADS) lut[i] = __fdiv_rn((float)i, 255.0f);
    const int W = p.w, H = p.h;
    const int x0 = bx * TS, y0 = by * TS;
    const int gx0 = x0 - GH, gy0 = y0 - GH;
    const float kw[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};
    __syncthreads();
    for (int k = threadIdx.x; k < RG * RG; k += SP_THREADS) {
        const int ly = k / RG, lx = k % RG;
        const int gx = gx0 + lx, gy = gy0 + ly;
        float v = 0.f;
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            const long long pi = (long long)gy * W + gx;
            float r, g, b;
            load_rgb(p, lut, pi, r, g, b);
            const float I = pi < p.vec_end ? luma_vec(r, g, b) : luma_tail(r, g, b);
            v = __fadd_rn(p.gray_out[pi], -I);
        }
        P[ly][lx] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < RG * TS; k += SP_THREADS) {
        const int ly = k / TS, tx = k % TS;
        const int gx = x0 + tx, gy = gy0 + ly;
        if (gx >= W || gy < 0 || gy >= H) continue;
        float s = 0.f, wsum = 0.f;
#pragma unroll
        for (int d = -2; d <= 2; d++) {
            const int xx = gx + d;
            if (xx >= 0 && xx < W) {
                s = __fmaf_rn(P[ly][xx - gx0], kw[d + 2], s);
                wsum = __fadd_rn(wsum, kw[d + 2]);
            }
        }
        T[ly][tx] = __fdiv_rn(s, wsum);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < TS * TS; k += SP_THREADS) {
        const int ty = k / TS, tx = k % TS;
        const int gx = x0 + tx, gy = y0 + ty;
        if (gx >= W || gy >= H) continue;
        float s = 0.f, wsum = 0.f;
#pragma unroll
        for (int d = -2; d <= 2; d++) {
            const int yy = gy + d;
            if (yy >= 0 && yy < H) {
                s = __fmaf_rn(T[yy - gy0][tx], kw[d + 2], s);
                wsum = __fadd_rn(wsum, kw[d + 2]);
            }
        }
        const float dy = __fdiv_rn(s, wsum);
        const long long pi = (long long)gy * W + gx;
        float r, g, b;
        load_rgb(p, lut, pi, r, g, b);
        store_rgb(p, pi, r, g, b, dy);
    }
}

__global__ void __launch_bounds__(SP_THREADS) k_guided_transfer(SpArgs args) {
    guided_body(args.p, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(SP_THREADS) k_gauss_transfer(SpArgs args) {
    gauss_body(args.p, blockIdx.x, blockIdx.y);
}
// batched: task = one stream (edge-aware and Gaussian streams in separate launches)
__global__ void __launch_bounds__(SP_THREADS)
    k_guided_transfer_multi(const TransferParams* __restrict__ ps, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    guided_body(ps[t.task], t.x, t.y);
}
__global__ void __launch_bounds__(SP_THREADS)
    k_gauss_transfer_multi(const TransferParams* __restrict__ ps, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    gauss_body(ps[t.task], t.x, t.y);
}

__global__ void k_passthrough(SpArgs args) {
    const TransferParams& p = args.p;
    const long long n = (long long)p.w * p.h * 3;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float v = p.src_u8 ? __fdiv_rn((float)p.src_u8[i], 255.0f) : p.src_f32[i];
        if (p.out_u8) p.out_u8[i] = p.src_u8 ? p.src_u8[i] : quant_u8(v);
        if (p.out_f32) p.out_f32[i] = v;
    }
}

cudaError_t spatial_prepare_device() {
    cudaError_t e = cudaFuncSetAttribute(k_guided_transfer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(GuidedSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guided_transfer_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(GuidedSmem));
    return e;
}

unsigned transfer_grid(const TransferParams& p, unsigned& gx, unsigned& gy) {
    gx = (unsigned)((p.w + TS - 1) / TS);
    gy = (unsigned)((p.h + TS - 1) / TS);
    return gx * gy;
}

cudaError_t launch_transfer_multi(int edge_aware, const TransferParams* d_params, const int* d_map,
                                  unsigned blocks, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    if (edge_aware)
        k_guided_transfer_multi<<<blocks, SP_THREADS, sizeof(GuidedSmem), st>>>(d_params, d_map);
    else
        k_gauss_transfer_multi<<<blocks, SP_THREADS, 0, st>>>(d_params, d_map);
    return cudaGetLastError();
}

cudaError_t launch_transfer(const TransferParams& p, cudaStream_t st) {
    SpArgs a{p};
    dim3 grid((p.w + TS - 1) / TS, (p.h + TS - 1) / TS);
    if (p.edge_aware) k_guided_transfer<<<grid, SP_THREADS, sizeof(GuidedSmem), st>>>(a);
    else k_gauss_transfer<<<grid, SP_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_passthrough(const TransferParams& p, cudaStream_t st) {
    SpArgs a{p};
    const long long n = (long long)p.w * p.h * 3;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_passthrough<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace wema
