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
// reference's definition), computed here by window sums sliding along short
// segments in shared memory rather than by the reference's FP32 running
// prefix sums - the two differ in the last bits only, which the u8 output
// absorbs (<= 1 LSB).
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

// Shared-memory rows are padded to 16-byte strides that keep 128-bit accesses
// by 8 consecutive rows on distinct banks; arrays dead after one phase share
// space with the next phase's.
constexpr int IS = 52;                  // row stride of I, p
constexpr int HS = 44;                  // row stride of the first-round row means and a, b
constexpr int QS = 36;                  // row stride of the second-round row means and dy
constexpr int NG = R0 * R0 / 4;         // 4-pixel groups of the 48x48 region (12 per row)

struct GuidedSmem {
    float I[R0][IS];                    // guide over the 48x48 region, 0 outside the image
    union {
        float P[R0][IS];                // p over the region (load, first-round rows)
        struct {
            float A[R1][HS];            // a, b over the 40x40 first-round region (0 outside)
            float B[R1][HS];
        } ab;
    } x;
    union {
        float hm[4][R0][HS];            // row means of I, p, I*I, I*p (0 outside the image)
        struct {
            float ha[2][R1][QS];        // row means of a, b
            float dy[TS][QS];           // the smoothed luma delta of the tile
        } sec;
    } y;
    uint32_t rgbw[TS][TS * 3 / 4];      // the tile's input RGB24 as words (word-aligned frames)
    float rcp[16];                      // 1/k for the clipped window counts k = 1 .. 2 GR + 1
    float lut[256];                     // u8 -> float, i / 255 correctly rounded
};

// 1 / (clipped count of a radius-4 window at coordinate c of a line of n)
__device__ __forceinline__ float inv_count(const float* rcp, int c, int n) {
    return rcp[min(c + GR, n - 1) - max(c - GR, 0) + 1];
}

__device__ __forceinline__ float byte_f(const float* lut, uint32_t w, int k) {
    return lut[(w >> (8 * k)) & 0xffu];
}

// guide luma of 4 pixels from their 12 RGB24 bytes (words a0 a1 a2); pi = first pixel
__device__ __forceinline__ void luma4(const float* lut, uint32_t a0, uint32_t a1, uint32_t a2,
                                      long long pi, long long vec_end, float v[4]) {
    float r[4], g[4], b[4];
    r[0] = byte_f(lut, a0, 0); g[0] = byte_f(lut, a0, 1); b[0] = byte_f(lut, a0, 2);
    r[1] = byte_f(lut, a0, 3); g[1] = byte_f(lut, a1, 0); b[1] = byte_f(lut, a1, 1);
    r[2] = byte_f(lut, a1, 2); g[2] = byte_f(lut, a1, 3); b[2] = byte_f(lut, a2, 0);
    r[3] = byte_f(lut, a2, 1); g[3] = byte_f(lut, a2, 2); b[3] = byte_f(lut, a2, 3);
    if (pi + 3 < vec_end) {
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = luma_vec(r[j], g[j], b[j]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
            v[j] = pi + j < vec_end ? luma_vec(r[j], g[j], b[j]) : luma_tail(r[j], g[j], b[j]);
    }
}

// Box means with the image's edges: every array holds 0 outside the image,
// so a radius-4 window's sum is its clipped sum, and the mean is that sum
// times 1/(clipped count).  Sums slide along segments of 8 (the last round 4)
// outputs.  Frames whose RGB24 rows are word-aligned (width a multiple of 4)
// move 4 pixels = 3 words per thread and access.  IN: the 48x48 region lies
// inside the image, so no test is needed and every count is 9.
template <bool IN>
__device__ __forceinline__ void guided_tile(const TransferParams& p, GuidedSmem& S, int bx, int by) {
    const int W = p.w, H = p.h;
    const int x0 = bx * TS, y0 = by * TS;
    const int gx0 = x0 - H0, gy0 = y0 - H0;      // region origin (may be negative)
    const int tid = threadIdx.x;
    const bool fast = p.src_u8 && !(W & 3) && !(reinterpret_cast<uintptr_t>(p.src_u8) & 3) &&
                      !(reinterpret_cast<uintptr_t>(p.gray_out) & 15);

    // region loads first (a thread's groups tid, tid + 256, tid + 512), tables meanwhile
    uint32_t wv[3][3];
    float4 gv[3];
    bool ok[3];
    if (fast) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int k = tid + i * SP_THREADS;
            const int ly = k / 12, g = k - ly * 12;
            const int gx = gx0 + 4 * g, gy = gy0 + ly;
            ok[i] = k < NG && (IN || (gx >= 0 && gx < W && gy >= 0 && gy < H));
            if (ok[i]) {
                const int pi = gy * W + gx;
                const uint32_t* q = reinterpret_cast<const uint32_t*>(p.src_u8) + 3 * (pi >> 2);
                wv[i][0] = __ldg(q);
                wv[i][1] = __ldg(q + 1);
                wv[i][2] = __ldg(q + 2);
                gv[i] = __ldg(reinterpret_cast<const float4*>(p.gray_out + pi));
            }
        }
    }
    S.lut[tid] = __fdiv_rn((float)tid, 255.0f);
    if (tid < 16) S.rcp[tid] = tid ? __frcp_rn((float)tid) : 0.f;
    __syncthreads();

    // I and p over the 48x48 region
    if (fast) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int k = tid + i * SP_THREADS;
            if (k >= NG) break;
            const int ly = k / 12, g = k - ly * 12;
            float4 Iv = make_float4(0.f, 0.f, 0.f, 0.f), Pv = Iv;
            if (ok[i]) {
                const uint32_t a0 = wv[i][0], a1 = wv[i][1], a2 = wv[i][2];
                float v[4];
                luma4(S.lut, a0, a1, a2, (long long)(gy0 + ly) * W + gx0 + 4 * g, p.vec_end, v);
                Iv = make_float4(v[0], v[1], v[2], v[3]);
                Pv = make_float4(__fadd_rn(gv[i].x, -v[0]), __fadd_rn(gv[i].y, -v[1]),
                                 __fadd_rn(gv[i].z, -v[2]), __fadd_rn(gv[i].w, -v[3]));
                const int ty = ly - H0, tg = g - H0 / 4;
                if (ty >= 0 && ty < TS && tg >= 0 && tg < TS / 4) {
                    S.rgbw[ty][3 * tg] = a0;
                    S.rgbw[ty][3 * tg + 1] = a1;
                    S.rgbw[ty][3 * tg + 2] = a2;
                }
            }
            *reinterpret_cast<float4*>(&S.I[ly][4 * g]) = Iv;
            *reinterpret_cast<float4*>(&S.x.P[ly][4 * g]) = Pv;
        }
    } else {
        for (int k = tid; k < R0 * R0; k += SP_THREADS) {
            const int ly = k / R0, lx = k - ly * R0;
            const int gx = gx0 + lx, gy = gy0 + ly;
            float I = 0.f, P = 0.f;
            if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
                const int pi = gy * W + gx;
                float r, g, b;
                load_rgb(p, S.lut, pi, r, g, b);
                I = pi < p.vec_end ? luma_vec(r, g, b) : luma_tail(r, g, b);
                P = __fadd_rn(p.gray_out[pi], -I);
            }
            S.I[ly][lx] = I;
            S.x.P[ly][lx] = P;
        }
    }
    __syncthreads();

    // first round, rows: 48 rows x 5 segments of 8 of the 40 columns
    if (tid < R0 * (R1 / 8)) {
        const int ly = tid % R0, c0 = (tid / R0) * 8;
        const int gy = gy0 + ly;
        const bool rowin = IN || (gy >= 0 && gy < H);
        const float r9 = S.rcp[2 * GR + 1];
        float Iv[16], Pv[16];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float4 a = *reinterpret_cast<const float4*>(&S.I[ly][c0 + 4 * j]);
            const float4 b = *reinterpret_cast<const float4*>(&S.x.P[ly][c0 + 4 * j]);
            Iv[4 * j] = a.x; Iv[4 * j + 1] = a.y; Iv[4 * j + 2] = a.z; Iv[4 * j + 3] = a.w;
            Pv[4 * j] = b.x; Pv[4 * j + 1] = b.y; Pv[4 * j + 2] = b.z; Pv[4 * j + 3] = b.w;
        }
        float sI = 0.f, sP = 0.f, sII = 0.f, sIP = 0.f;
        // output column cx sits at region column cx + GR; its window is cx .. cx + 2 GR
#pragma unroll
        for (int x = 0; x < 2 * GR; x++) {
            sI = __fadd_rn(sI, Iv[x]);
            sP = __fadd_rn(sP, Pv[x]);
            sII = __fmaf_rn(Iv[x], Iv[x], sII);
            sIP = __fmaf_rn(Iv[x], Pv[x], sIP);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float o[4][4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int x = 4 * h + j;
                const float In = Iv[x + 2 * GR], Pn = Pv[x + 2 * GR];
                sI = __fadd_rn(sI, In);
                sP = __fadd_rn(sP, Pn);
                sII = __fmaf_rn(In, In, sII);
                sIP = __fmaf_rn(In, Pn, sIP);
                const int gx = x0 - GR + c0 + x;
                const bool in = IN || (rowin && gx >= 0 && gx < W);
                const float inv = IN ? r9 : inv_count(S.rcp, gx, W);
                o[0][j] = in ? __fmul_rn(sI, inv) : 0.f;
                o[1][j] = in ? __fmul_rn(sP, inv) : 0.f;
                o[2][j] = in ? __fmul_rn(sII, inv) : 0.f;
                o[3][j] = in ? __fmul_rn(sIP, inv) : 0.f;
                sI = __fsub_rn(sI, Iv[x]);
                sP = __fsub_rn(sP, Pv[x]);
                sII = __fmaf_rn(-Iv[x], Iv[x], sII);
                sIP = __fmaf_rn(-Iv[x], Pv[x], sIP);
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<float4*>(&S.y.hm[q][ly][c0 + 4 * h]) =
                    make_float4(o[q][0], o[q][1], o[q][2], o[q][3]);
        }
    }
    __syncthreads();

    // first round, columns -> a, b: 40 columns x 5 segments of 8 of the 40 rows
    if (tid < R1 * (R1 / 8)) {
        const int cx = tid % R1, r0 = (tid / R1) * 8;
        const int gx = x0 - GR + cx;
        const bool colin = IN || (gx >= 0 && gx < W);
        const float r9 = S.rcp[2 * GR + 1];
        float m[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int y = r0; y < r0 + 2 * GR; y++)
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fadd_rn(m[q], S.y.hm[q][y][cx]);
        float av[8], bv[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int cy = r0 + j;
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fadd_rn(m[q], S.y.hm[q][cy + 2 * GR][cx]);
            const int gy = y0 - GR + cy;
            av[j] = 0.f;
            bv[j] = 0.f;
            if (IN || (colin && gy >= 0 && gy < H)) {
                const float inv = IN ? r9 : inv_count(S.rcp, gy, H);
                const float mI = __fmul_rn(m[0], inv), mP = __fmul_rn(m[1], inv);
                const float cII = __fmul_rn(m[2], inv), cIP = __fmul_rn(m[3], inv);
                // the denominator is >= 0.01 - mI^2 + E[I^2] > 0; a within 2 ulp
                av[j] = __fdividef(__fmaf_rn(-mI, mP, cIP), __fmaf_rn(-mI, mI, __fadd_rn(cII, 0.01f)));
                bv[j] = __fmaf_rn(-av[j], mI, mP);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) m[q] = __fsub_rn(m[q], S.y.hm[q][cy][cx]);
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            S.x.ab.A[r0 + j][cx] = av[j];
            S.x.ab.B[r0 + j][cx] = bv[j];
        }
    }
    __syncthreads();

    // second round, rows: 40 rows x 4 segments of 8 of the tile's 32 columns
    if (tid < R1 * (TS / 8)) {
        const int cy = tid % R1, t0 = (tid / R1) * 8;
        const float r9 = S.rcp[2 * GR + 1];
        float Av[16], Bv[16];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float4 a = *reinterpret_cast<const float4*>(&S.x.ab.A[cy][t0 + 4 * j]);
            const float4 b = *reinterpret_cast<const float4*>(&S.x.ab.B[cy][t0 + 4 * j]);
            Av[4 * j] = a.x; Av[4 * j + 1] = a.y; Av[4 * j + 2] = a.z; Av[4 * j + 3] = a.w;
            Bv[4 * j] = b.x; Bv[4 * j + 1] = b.y; Bv[4 * j + 2] = b.z; Bv[4 * j + 3] = b.w;
        }
        float sa = 0.f, sb = 0.f;
        // tile column tx sits at first-round column tx + GR; window tx .. tx + 2 GR
#pragma unroll
        for (int x = 0; x < 2 * GR; x++) {
            sa = __fadd_rn(sa, Av[x]);
            sb = __fadd_rn(sb, Bv[x]);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float oa[4], ob[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int x = 4 * h + j;
                sa = __fadd_rn(sa, Av[x + 2 * GR]);
                sb = __fadd_rn(sb, Bv[x + 2 * GR]);
                const float inv = IN ? r9 : inv_count(S.rcp, min(x0 + t0 + x, W - 1), W);
                oa[j] = __fmul_rn(sa, inv);
                ob[j] = __fmul_rn(sb, inv);
                sa = __fsub_rn(sa, Av[x]);
                sb = __fsub_rn(sb, Bv[x]);
            }
            *reinterpret_cast<float4*>(&S.y.sec.ha[0][cy][t0 + 4 * h]) = make_float4(oa[0], oa[1], oa[2], oa[3]);
            *reinterpret_cast<float4*>(&S.y.sec.ha[1][cy][t0 + 4 * h]) = make_float4(ob[0], ob[1], ob[2], ob[3]);
        }
    }
    __syncthreads();

    // second round, columns -> dy: 32 columns x 8 segments of 4 rows
    {
        const int tx = tid % TS, t0 = (tid / TS) * 4;
        const float r9 = S.rcp[2 * GR + 1];
        float sa = 0.f, sb = 0.f;
#pragma unroll
        for (int y = t0; y < t0 + 2 * GR; y++) {
            sa = __fadd_rn(sa, S.y.sec.ha[0][y][tx]);
            sb = __fadd_rn(sb, S.y.sec.ha[1][y][tx]);
        }
        float d[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int ty = t0 + j;
            sa = __fadd_rn(sa, S.y.sec.ha[0][ty + 2 * GR][tx]);
            sb = __fadd_rn(sb, S.y.sec.ha[1][ty + 2 * GR][tx]);
            const float inv = IN ? r9 : inv_count(S.rcp, min(y0 + ty, H - 1), H);
            d[j] = __fmaf_rn(__fmul_rn(sa, inv), S.I[ty + H0][tx + H0], __fmul_rn(sb, inv));
            sa = __fsub_rn(sa, S.y.sec.ha[0][ty][tx]);
            sb = __fsub_rn(sb, S.y.sec.ha[1][ty][tx]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) S.y.sec.dy[t0 + j][tx] = d[j];
    }
    __syncthreads();

    // out = clamp01(RGB + dy): a thread per 4-pixel group of the tile where the
    // frame layout allows, else per pixel
    const bool fast_out = fast && !(reinterpret_cast<uintptr_t>(p.out_u8) & 3) &&
                          !(reinterpret_cast<uintptr_t>(p.out_f32) & 15);
    if (fast_out) {
        const int ty = tid >> 3, g = tid & 7;
        const int gx = x0 + 4 * g, gy = y0 + ty;
        if (IN || (gx < W && gy < H)) {
            const int pi = gy * W + gx;
            const float4 dv = *reinterpret_cast<const float4*>(&S.y.sec.dy[ty][4 * g]);
            const float dyv[4] = {dv.x, dv.y, dv.z, dv.w};
            const uint32_t w[3] = {S.rgbw[ty][3 * g], S.rgbw[ty][3 * g + 1], S.rgbw[ty][3 * g + 2]};
            float v[12];
            uint32_t ow[3] = {0u, 0u, 0u};
#pragma unroll
            for (int c = 0; c < 12; c++) {
                v[c] = clamp01(__fadd_rn(byte_f(S.lut, w[c >> 2], c & 3), dyv[c / 3]));
                ow[c >> 2] |= (uint32_t)quant_u8(v[c]) << (8 * (c & 3));
            }
            if (p.out_u8) {
                uint32_t* d = reinterpret_cast<uint32_t*>(p.out_u8) + 3 * (pi >> 2);
                d[0] = ow[0];
                d[1] = ow[1];
                d[2] = ow[2];
            }
            if (p.out_f32) {
                float4* d = reinterpret_cast<float4*>(p.out_f32 + 3 * (long long)pi);
                d[0] = make_float4(v[0], v[1], v[2], v[3]);
                d[1] = make_float4(v[4], v[5], v[6], v[7]);
                d[2] = make_float4(v[8], v[9], v[10], v[11]);
            }
        }
    } else {
        for (int k = tid; k < TS * TS; k += SP_THREADS) {
            const int ty = k / TS, tx = k - ty * TS;
            const int gx = x0 + tx, gy = y0 + ty;
            if (gx >= W || gy >= H) continue;
            const int pi = gy * W + gx;
            float r, g, b;
            load_rgb(p, S.lut, pi, r, g, b);
            store_rgb(p, pi, r, g, b, S.y.sec.dy[ty][tx]);
        }
    }
}

__device__ __forceinline__ void guided_body(const TransferParams& p, int bx, int by) {
    extern __shared__ __align__(16) unsigned char raw[];
    GuidedSmem& S = *reinterpret_cast<GuidedSmem*>(raw);
    const int gx0 = bx * TS - H0, gy0 = by * TS - H0;
    if (gx0 >= 0 && gy0 >= 0 && gx0 + R0 <= p.w && gy0 + R0 <= p.h) guided_tile<true>(p, S, bx, by);
    else guided_tile<false>(p, S, bx, by);
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
