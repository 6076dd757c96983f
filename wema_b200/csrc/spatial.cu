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

__device__ __forceinline__ void load_rgb(const TransferParams& p, const float* lut, int pi,
                                         float& r, float& g, float& b) {
    if (p.src_u8) {
        const uint8_t* q = p.src_u8 + 3 * pi;
        r = lut[q[0]]; g = lut[q[1]]; b = lut[q[2]];
    } else {
        const float* q = p.src_f32 + 3 * pi;
        r = q[0]; g = q[1]; b = q[2];
    }
}

__device__ __forceinline__ void store_rgb(const TransferParams& p, int pi, float r, float g,
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
    float I[R0][R0 + 1];          // guide and p over the 48x48 region, 0 outside the image
    float P[R0][R0 + 1];
    float hm[4][R0][R1 + 1];      // row means of I, p, I*I, I*p (rows outside the image: 0)
    float A[R1][R1 + 1];          // a, b over the 40x40 first-round region (0 outside)
    float B[R1][R1 + 1];
    float ha[2][R1][TS + 1];      // row means of a, b
    float dy[TS][TS + 1];         // the smoothed luma delta of the tile
    float rgb[TS][TS][3];         // the tile's input RGB (reused by the output pass)
    float rcp[2 * GR + 2];        // 1/k for the clipped window counts k = 1 .. 2 GR + 1
};

// 1 / (clipped count of a radius-4 window at coordinate c of a line of n)
__device__ __forceinline__ float inv_count(const float* rcp, int c, int n) {
    return rcp[min(c + GR, n - 1) - max(c - GR, 0) + 1];
}

// Box means with the image's edges: every array holds 0 outside the image,
// so a radius-4 window's sum is its clipped sum, and the mean is that sum
// times 1/(clipped count).  Sums slide along segments of 8 outputs.
__device__ __forceinline__ void guided_body(const TransferParams& p, int bx, int by) {
    extern __shared__ unsigned char raw[];
    GuidedSmem& S = *reinterpret_cast<GuidedSmem*>(raw);
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += SP_THREADS) lut[i] = __fdiv_rn((float)i, 255.0f);
    if (threadIdx.x < 2 * GR + 2) S.rcp[threadIdx.x] = threadIdx.x ? __frcp_rn((float)threadIdx.x) : 0.f;
    const int W = p.w, H = p.h;
    const int x0 = bx * TS, y0 = by * TS;
    const int gx0 = x0 - H0, gy0 = y0 - H0;      // region origin (may be negative)
    __syncthreads();

    // I and p over the 48x48 region
    for (int k = threadIdx.x; k < R0 * R0; k += SP_THREADS) {
        const int ly = k / R0, lx = k - ly * R0;
        const int gx = gx0 + lx, gy = gy0 + ly;
        float I = 0.f, P = 0.f;
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            const int pi = gy * W + gx;
            float r, g, b;
            load_rgb(p, lut, pi, r, g, b);
            I = pi < p.vec_end ? luma_vec(r, g, b) : luma_tail(r, g, b);
            P = __fadd_rn(p.gray_out[pi], -I);
            const int ty = ly - H0, tx = lx - H0;
            if (ty >= 0 && ty < TS && tx >= 0 && tx < TS) {
                S.rgb[ty][tx][0] = r;
                S.rgb[ty][tx][1] = g;
                S.rgb[ty][tx][2] = b;
            }
        }
        S.I[ly][lx] = I;
        S.P[ly][lx] = P;
    }
    __syncthreads();

    // first round, rows: 48 rows x 5 segments of 8 of the 40 columns
    if (threadIdx.x < R0 * (R1 / 8)) {
        const int ly = threadIdx.x / (R1 / 8), c0 = (threadIdx.x % (R1 / 8)) * 8;
        const int gy = gy0 + ly;
        const float* Ir = S.I[ly];
        const float* Pr = S.P[ly];
        float sI = 0.f, sP = 0.f, sII = 0.f, sIP = 0.f;
        // output column cx sits at region column cx + GR; its window is cx .. cx + 2 GR
#pragma unroll
        for (int x = c0; x < c0 + 2 * GR; x++) {
            const float I = Ir[x], P = Pr[x];
            sI = __fadd_rn(sI, I);
            sP = __fadd_rn(sP, P);
            sII = __fmaf_rn(I, I, sII);
            sIP = __fmaf_rn(I, P, sIP);
        }
#pragma unroll
        for (int cx = c0; cx < c0 + 8; cx++) {
            const float In = Ir[cx + 2 * GR], Pn = Pr[cx + 2 * GR];
            sI = __fadd_rn(sI, In);
            sP = __fadd_rn(sP, Pn);
            sII = __fmaf_rn(In, In, sII);
            sIP = __fmaf_rn(In, Pn, sIP);
            const int gx = x0 - GR + cx;
            const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
            const float inv = inv_count(S.rcp, gx, W);
            S.hm[0][ly][cx] = in ? __fmul_rn(sI, inv) : 0.f;
            S.hm[1][ly][cx] = in ? __fmul_rn(sP, inv) : 0.f;
            S.hm[2][ly][cx] = in ? __fmul_rn(sII, inv) : 0.f;
            S.hm[3][ly][cx] = in ? __fmul_rn(sIP, inv) : 0.f;
            const float Io = Ir[cx], Po = Pr[cx];
            sI = __fsub_rn(sI, Io);
            sP = __fsub_rn(sP, Po);
            sII = __fmaf_rn(-Io, Io, sII);
            sIP = __fmaf_rn(-Io, Po, sIP);
        }
    }
    __syncthreads();

    // first round, columns -> a, b: 40 columns x 5 segments of 8 of the 40 rows
    if (threadIdx.x < R1 * (R1 / 8)) {
        const int cx = threadIdx.x / (R1 / 8), r0 = (threadIdx.x % (R1 / 8)) * 8;
        const int gx = x0 - GR + cx;
        float m[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int y = r0; y < r0 + 2 * GR; y++)
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fadd_rn(m[q], S.hm[q][y][cx]);
#pragma unroll
        for (int cy = r0; cy < r0 + 8; cy++) {
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fadd_rn(m[q], S.hm[q][cy + 2 * GR][cx]);
            const int gy = y0 - GR + cy;
            float av = 0.f, bv = 0.f;
            if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
                const float inv = inv_count(S.rcp, gy, H);
                const float mI = __fmul_rn(m[0], inv), mP = __fmul_rn(m[1], inv);
                const float cII = __fmul_rn(m[2], inv), cIP = __fmul_rn(m[3], inv);
                av = __fdiv_rn(__fmaf_rn(-mI, mP, cIP), __fmaf_rn(-mI, mI, __fadd_rn(cII, 0.01f)));
                bv = __fmaf_rn(-av, mI, mP);
            }
            S.A[cy][cx] = av;
            S.B[cy][cx] = bv;
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fsub_rn(m[q], S.hm[q][cy][cx]);
        }
    }
    __syncthreads();

    // second round, rows: 40 rows x 4 segments of 8 of the tile's 32 columns
    if (threadIdx.x < R1 * (TS / 8)) {
        const int cy = threadIdx.x / (TS / 8), t0 = (threadIdx.x % (TS / 8)) * 8;
        float sa = 0.f, sb = 0.f;
        // tile column tx sits at first-round column tx + GR; window tx .. tx + 2 GR
#pragma unroll
        for (int x = t0; x < t0 + 2 * GR; x++) {
            sa = __fadd_rn(sa, S.A[cy][x]);
            sb = __fadd_rn(sb, S.B[cy][x]);
        }
#pragma unroll
        for (int tx = t0; tx < t0 + 8; tx++) {
            sa = __fadd_rn(sa, S.A[cy][tx + 2 * GR]);
            sb = __fadd_rn(sb, S.B[cy][tx + 2 * GR]);
            const float inv = inv_count(S.rcp, min(x0 + tx, W - 1), W);
            S.ha[0][cy][tx] = __fmul_rn(sa, inv);
            S.ha[1][cy][tx] = __fmul_rn(sb, inv);
            sa = __fsub_rn(sa, S.A[cy][tx]);
            sb = __fsub_rn(sb, S.B[cy][tx]);
        }
    }
    __syncthreads();

    // second round, columns: 32 columns x 4 segments of 8 rows -> dy
    if (threadIdx.x < TS * (TS / 8)) {
        const int tx = threadIdx.x / (TS / 8), t0 = (threadIdx.x % (TS / 8)) * 8;
        float sa = 0.f, sb = 0.f;
#pragma unroll
        for (int y = t0; y < t0 + 2 * GR; y++) {
            sa = __fadd_rn(sa, S.ha[0][y][tx]);
            sb = __fadd_rn(sb, S.ha[1][y][tx]);
        }
#pragma unroll
        for (int ty = t0; ty < t0 + 8; ty++) {
            sa = __fadd_rn(sa, S.ha[0][ty + 2 * GR][tx]);
            sb = __fadd_rn(sb, S.ha[1][ty + 2 * GR][tx]);
            const float inv = inv_count(S.rcp, min(y0 + ty, H - 1), H);
            const float ma = __fmul_rn(sa, inv), mb = __fmul_rn(sb, inv);
            S.dy[ty][tx] = __fmaf_rn(ma, S.I[ty + H0][tx + H0], mb);
            sa = __fsub_rn(sa, S.ha[0][ty][tx]);
            sb = __fsub_rn(sb, S.ha[1][ty][tx]);
        }
    }
    __syncthreads();

    for (int k = threadIdx.x; k < TS * TS; k += SP_THREADS) {
        const int ty = k / TS, tx = k - ty * TS;
        const int gx = x0 + tx, gy = y0 + ty;
        if (gx >= W || gy >= H) continue;
        store_rgb(p, gy * W + gx, S.rgb[ty][tx][0], S.rgb[ty][tx][1], S.rgb[ty][tx][2], S.dy[ty][tx]);
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
