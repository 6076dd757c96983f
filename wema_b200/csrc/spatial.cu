// spatial.cu - luma-delta smoothing and transfer to RGB, fused with the u8
// output (wema.c:289-335, wema_batch.c:311-346).
//
// guide I = luma of the input frame (same evaluation as the DWT input),
// p = gray_out - I, smoothed by the guided filter (radius 4, eps 0.01,
// wema.c:173-230) or, with edge-aware off, the 5-tap [1 4 6 4 1]/16 blur
// with border renormalisation (wema.c:236-283); then
// out = clamp01(RGB + smooth) and u8 = (uint8)(v*255 + 0.5).
//
// Guided filter: one warp sweeps a strip of the frame from top to bottom
// (see guided_sweep).  Every box mean is the clipped window's sum divided by
// the clipped count (the reference's definition); the sums here are
// vertical running sums over a 9-row ring and horizontal window sums across
// the warp's lanes, not the reference's FP32 running prefix sums - the two
// differ in the last bits only, which the u8 output absorbs (<= 1 LSB).
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

#include <algorithm>
#include <atomic>

namespace wema {

constexpr int TS = 32;                  // Gaussian fallback: output tile
constexpr int SP_THREADS = 256;         // Gaussian fallback: threads per tile

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

// ---- guided filter: a vertical sweep per warp --------------------------------
//
// A warp owns a strip of 128 input columns, 4 consecutive columns per lane,
// and sweeps a segment of `seg_rows` output rows from top to bottom.  The
// strip's first and last 8 columns are the halo of the two radius-4 rounds,
// so a strip produces 112 output columns (lanes 2..29); strips overlap by 16
// columns and segments by 16 rows (the vertical halo), about 1.14 x 1.13
// the output area loaded, against 2.25 for a 32x32 tile with its 8-pixel
// border.  Per input row r entering the sweep:
//   I, p of row r (0 outside the image) go into a 9-row ring in shared
//   memory; vertical running sums of I, p, I*I, I*p over rows r-8..r add
//   row r and drop row r-9 (read back from the ring);
//   the first round at row r-4: horizontal 9-column window sums of those
//   vertical sums, exchanged with the neighbouring lanes by shuffles, times
//   1/(clipped column count x clipped row count) give mean_I, mean_p,
//   corr_II, corr_Ip and then a, b (0 outside the image, wema.c:206-217);
//   the horizontal window sums of a and b go into a second 9-row ring, whose
//   vertical running sums over rows r-12..r-4 give the second round at row
//   r-8: dy = mean_a * I + mean_b (wema.c:218-229, I read back from the
//   first ring), added to the row's RGB, clamped and quantised.
// Every running sum is recomputed from its ring, oldest row first, at rows
// fixed in the frame (first round: window ends r = 0 mod 16; second round:
// c1 = 4 mod 16) and slides from there, so a row's sums do not depend on
// where its segment starts: any seg_rows that is a multiple of 16 gives
// bit-identical output, and rounding drift spans at most 15 slides.
constexpr int GR = 4;                   // guided-filter radius (wema.c:314)
constexpr int GS_IN = 128;              // input columns per strip (4 per lane)
constexpr int GS_OUT = GS_IN - 4 * GR;  // output columns per strip
constexpr int GS_RING = 2 * GR + 1;     // rows in each ring
constexpr int GS_WARPS = 2;             // strips per CTA (one per warp)
constexpr int GS_THREADS = 32 * GS_WARPS;
constexpr int GS_ROWS_DEFAULT = 64;       // the autotuner's usual choice on B200
constexpr float kEps = 0.01f;           // wema.c:315
constexpr unsigned kFull = 0xffffffffu;

struct SweepRing {                      // one warp's rings
    float4 ip[GS_RING][2][32];          // I, p of rows r-8..r; lane l holds columns 4l..4l+3
    float4 ab[GS_RING][2][32];          // horizontal window sums of a, b
};

// 1/k for the clipped window counts k = 1 .. 2 GR + 1 (index 0 unused),
// correctly rounded (the compiler's IEEE division)
__constant__ float c_rcp[2 * GR + 2] = {0.f, 1.f / 1, 1.f / 2, 1.f / 3, 1.f / 4, 1.f / 5,
                                         1.f / 6, 1.f / 7, 1.f / 8, 1.f / 9};

// 1 / (clipped count of a radius-4 window at coordinate c of a line of n);
// 0 for c outside the line
__device__ __forceinline__ float inv_count(int c, int n) {
    if (c < 0 || c >= n) return 0.f;
    return c_rcp[min(c + GR, n - 1) - max(c - GR, 0) + 1];
}

// The 9-column window sums centred on a lane's 4 columns: its own 4 values
// and its neighbours' 4 each, by shuffles (lanes 0 and 31 get garbage, which
// only halo columns use).
__device__ __forceinline__ void hwin(const float v[4], float o[4]) {
    float L[4], R[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        L[j] = __shfl_up_sync(kFull, v[j], 1);
        R[j] = __shfl_down_sync(kFull, v[j], 1);
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(L[0], L[1]), __fadd_rn(L[2], L[3])),
                        __fadd_rn(__fadd_rn(v[0], v[1]), __fadd_rn(v[2], v[3])));
    s = __fadd_rn(s, R[0]);
    o[0] = s;
#pragma unroll
    for (int j = 1; j < 4; j++) {
        s = __fadd_rn(__fsub_rn(s, L[j - 1]), R[j]);
        o[j] = s;
    }
}

// One row of 4 pixels of a lane: the loads of row r (issued a row ahead) and
// their decoding.  FAST: RGB24 rows word-aligned (width a multiple of 4 and
// aligned buffers, frames below 2^29 pixels): the 4 pixels are 3 words, all in
// or all out of the image, and pixel, word and float indices fit 32 bits.
template <bool FAST>
struct RowLoad {
    uint32_t w[3];
    float4 g;
    float rgb[12];                      // generic path: decoded RGB
    float gv[4];
    uint32_t ow[3];                     // FAST: RGB words of row r - 2 GR, the step's output row
    bool any;

    __device__ __forceinline__ void issue(const TransferParams& p, int r, int cx) {
        any = r >= 0 && r < p.h && cx + 3 >= 0 && cx < p.w;
        if (FAST) {
            // the output row's words (loaded as input 2 GR rows earlier, so mostly
            // cache hits), issued a row ahead of their use like the input
            const int y = r - 2 * GR;
            if (y >= 0 && y < p.h && cx >= 0 && cx < p.w) {
                const uint32_t* q = reinterpret_cast<const uint32_t*>(p.src_u8) + 3 * ((y * p.w + cx) >> 2);
                ow[0] = __ldg(q);
                ow[1] = __ldg(q + 1);
                ow[2] = __ldg(q + 2);
            }
            if (any) {
                const int pi = r * p.w + cx;
                const uint32_t* q = reinterpret_cast<const uint32_t*>(p.src_u8) + 3 * (pi >> 2);
                w[0] = __ldg(q);
                w[1] = __ldg(q + 1);
                w[2] = __ldg(q + 2);
                if (p.h16) {
                    const uint2 hb = __ldg(reinterpret_cast<const uint2*>(
                        reinterpret_cast<const __half*>(p.gray_out) + pi));
                    const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&hb.x));
                    const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&hb.y));
                    g = make_float4(lo.x, lo.y, hi.x, hi.y);
                } else {
                    g = __ldg(reinterpret_cast<const float4*>(p.gray_out + pi));
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int x = cx + j;
                const bool in = any && x >= 0 && x < p.w;
                const long long pi = (long long)r * p.w + x;
                gv[j] = in ? pl_ld(p.gray_out, pi, p.h16) : 0.f;
#pragma unroll
                for (int c = 0; c < 3; c++)
                    rgb[3 * j + c] = !in ? 0.f
                                         : (p.src_u8 ? u8f(__ldg(p.src_u8 + 3 * pi + c))
                                                     : __ldg(p.src_f32 + 3 * pi + c));
            }
        }
    }

    // guide I and p = gray_out - I of the 4 pixels (0 outside the image)
    __device__ __forceinline__ void decode(const TransferParams& p, int r, int cx, float I[4],
                                           float P[4]) const {
        float rr[4], gg[4], bb[4], gy[4];
        if (FAST) {
            rr[0] = byte_of(w[0], 0); gg[0] = byte_of(w[0], 1); bb[0] = byte_of(w[0], 2);
            rr[1] = byte_of(w[0], 3); gg[1] = byte_of(w[1], 0); bb[1] = byte_of(w[1], 1);
            rr[2] = byte_of(w[1], 2); gg[2] = byte_of(w[1], 3); bb[2] = byte_of(w[2], 0);
            rr[3] = byte_of(w[2], 1); gg[3] = byte_of(w[2], 2); bb[3] = byte_of(w[2], 3);
            gy[0] = g.x; gy[1] = g.y; gy[2] = g.z; gy[3] = g.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                rr[j] = rgb[3 * j]; gg[j] = rgb[3 * j + 1]; bb[j] = rgb[3 * j + 2];
                gy[j] = gv[j];
            }
        }
        float Iv[4];
        const long long pi0 = (long long)r * p.w + cx;
        // all four in the vector body: (FAST) every row but the last - the vector
        // body ends at most 3 pixels before the frame's end, and 4 | w
        if ((FAST && r + 1 < p.h) || pi0 + 3 < p.vec_end) {
#pragma unroll
            for (int j = 0; j < 4; j++) Iv[j] = luma_vec(rr[j], gg[j], bb[j]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                Iv[j] = pi0 + j < p.vec_end ? luma_vec(rr[j], gg[j], bb[j]) : luma_tail(rr[j], gg[j], bb[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool in = any && (FAST || (cx + j >= 0 && cx + j < p.w));
            I[j] = in ? Iv[j] : 0.f;
            P[j] = in ? __fadd_rn(gy[j], -Iv[j]) : 0.f;
        }
    }
};

// out = clamp01(RGB + dy) of a lane's 4 output pixels of row y
// (FAST: w holds the row's 3 RGB words of the lane's 4 pixels, loaded ahead)
template <bool FAST>
__device__ __forceinline__ void put_row(const TransferParams& p, int y, int cx, const float dy[4],
                                        const uint32_t (&w)[3]) {
    if (FAST) {
        if (cx < 0 || cx >= p.w) return;
        const int pi0 = y * p.w + cx;
        float v[12];
        uint32_t qb[12];
#pragma unroll
        for (int c = 0; c < 12; c++) {
            // clamp01 of a finite sum: the saturating add
            v[c] = __saturatef(__fadd_rn(byte_of(w[c >> 2], c & 3), dy[c / 3]));
            qb[c] = quant_bits(v[c]);
        }
        uint32_t ow[3];
#pragma unroll
        for (int k = 0; k < 3; k++)   // low bytes of four quantised values into one word
            ow[k] = __byte_perm(__byte_perm(qb[4 * k], qb[4 * k + 1], 0x0040u),
                                __byte_perm(qb[4 * k + 2], qb[4 * k + 3], 0x0040u), 0x5410u);
        if (p.out_u8) {
            uint32_t* d = reinterpret_cast<uint32_t*>(p.out_u8) + 3 * (pi0 >> 2);
            d[0] = ow[0];
            d[1] = ow[1];
            d[2] = ow[2];
        }
        if (p.out_f32) {
            float4* d = reinterpret_cast<float4*>(p.out_f32 + 3 * pi0);
            d[0] = make_float4(v[0], v[1], v[2], v[3]);
            d[1] = make_float4(v[4], v[5], v[6], v[7]);
            d[2] = make_float4(v[8], v[9], v[10], v[11]);
        }
    } else {
        const long long pi0 = (long long)y * p.w + cx;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int x = cx + j;
            if (x < 0 || x >= p.w) continue;
            const long long pi = pi0 + j;
            float c3[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float in = p.src_u8 ? u8f(__ldg(p.src_u8 + 3 * pi + c)) : __ldg(p.src_f32 + 3 * pi + c);
                c3[c] = clamp01(__fadd_rn(in, dy[j]));
            }
            if (p.out_u8) {
#pragma unroll
                for (int c = 0; c < 3; c++) p.out_u8[3 * pi + c] = quant_u8(c3[c]);
            }
            if (p.out_f32) {
#pragma unroll
                for (int c = 0; c < 3; c++) p.out_f32[3 * pi + c] = c3[c];
            }
        }
    }
}

template <bool FAST>
__device__ __forceinline__ void guided_sweep(const TransferParams& pg, SweepRing& R, int strip, int seg) {
    // the parameters in registers: read through the reference, every field the
    // loop uses would be loaded again after each output store, which may alias
    // the parameter table as far as the compiler knows (measured 0.58 -> 0.55 ms)
    const TransferParams p = pg;
    const int W = p.w, H = p.h;
    const int lane = threadIdx.x & 31;
    const int x0 = strip * GS_OUT;
    const int cx = x0 - 2 * GR + 4 * lane;          // this lane's first column
    const int ys = seg * p.seg_rows;
    const int ye = min(ys + p.seg_rows, H);
    if (x0 >= W || ys >= H) return;

    float icx[4];
#pragma unroll
    for (int j = 0; j < 4; j++) icx[j] = inv_count(cx + j, W);
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < GS_RING; k++) {
        R.ip[k][0][lane] = z4; R.ip[k][1][lane] = z4;
        R.ab[k][0][lane] = z4; R.ab[k][1][lane] = z4;
    }
    float vI[4] = {0.f, 0.f, 0.f, 0.f}, vP[4] = {0.f, 0.f, 0.f, 0.f};
    float vII[4] = {0.f, 0.f, 0.f, 0.f}, vIP[4] = {0.f, 0.f, 0.f, 0.f};
    float uA[4] = {0.f, 0.f, 0.f, 0.f}, uB[4] = {0.f, 0.f, 0.f, 0.f};
    int s1 = 0, s2 = 0;                             // ring slots of the row entering

    // one input row through the sweep (the row's loads were issued a row ahead)
    auto step = [&](const RowLoad<FAST>& in, int r) {
        float I[4], P[4];
        in.decode(p, r, cx, I, P);
        // ring of I, p; vertical sums over rows r-8..r
        {
            const float4 oI = R.ip[s1][0][lane], oP = R.ip[s1][1][lane];
            R.ip[s1][0][lane] = make_float4(I[0], I[1], I[2], I[3]);
            R.ip[s1][1][lane] = make_float4(P[0], P[1], P[2], P[3]);
            const float ofI[4] = {oI.x, oI.y, oI.z, oI.w}, ofP[4] = {oP.x, oP.y, oP.z, oP.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                vI[j] = __fsub_rn(__fadd_rn(vI[j], I[j]), ofI[j]);
                vP[j] = __fsub_rn(__fadd_rn(vP[j], P[j]), ofP[j]);
                vII[j] = __fmaf_rn(-ofI[j], ofI[j], __fmaf_rn(I[j], I[j], vII[j]));
                vIP[j] = __fmaf_rn(-ofI[j], ofP[j], __fmaf_rn(I[j], P[j], vIP[j]));
            }
            if ((r & 15) == 0) {                    // anchor: the window's sums afresh
#pragma unroll
                for (int j = 0; j < 4; j++) vI[j] = vP[j] = vII[j] = vIP[j] = 0.f;
#pragma unroll
                for (int k = 1; k <= GS_RING; k++) {   // slots s1+1 .. s1+9: rows r-8 .. r
                    const int sl = s1 + k < GS_RING ? s1 + k : s1 + k - GS_RING;
                    const float4 a4 = R.ip[sl][0][lane], b4 = R.ip[sl][1][lane];
                    const float ai[4] = {a4.x, a4.y, a4.z, a4.w}, bi[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        vI[j] = __fadd_rn(vI[j], ai[j]);
                        vP[j] = __fadd_rn(vP[j], bi[j]);
                        vII[j] = __fmaf_rn(ai[j], ai[j], vII[j]);
                        vIP[j] = __fmaf_rn(ai[j], bi[j], vIP[j]);
                    }
                }
            }
            s1 = s1 == GS_RING - 1 ? 0 : s1 + 1;
        }
        if (r < ys) return;                         // rows r-8..r not all in yet
        // first round at row c1 = r - 4: a, b
        float a[4], b[4];
        {
            float sI[4], sP[4], sII[4], sIP[4];
            hwin(vI, sI);
            hwin(vP, sP);
            hwin(vII, sII);
            hwin(vIP, sIP);
            const float icy = inv_count(r - GR, H);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float inv = __fmul_rn(icx[j], icy);
                const float mI = __fmul_rn(sI[j], inv), mP = __fmul_rn(sP[j], inv);
                const float cII = __fmul_rn(sII[j], inv), cIP = __fmul_rn(sIP[j], inv);
                // the denominator is >= eps + E[I^2] - E[I]^2 > 0; a within 2 ulp
                const float av = __fdividef(__fmaf_rn(-mI, mP, cIP),
                                            __fmaf_rn(-mI, mI, __fadd_rn(cII, kEps)));
                const bool inside = inv != 0.f;
                a[j] = inside ? av : 0.f;
                b[j] = inside ? __fmaf_rn(-av, mI, mP) : 0.f;
            }
        }
        // second round: horizontal sums of a, b into the ring; vertical sums over rows c1-8..c1
        {
            float hA[4], hB[4];
            hwin(a, hA);
            hwin(b, hB);
            const float4 oA = R.ab[s2][0][lane], oB = R.ab[s2][1][lane];
            R.ab[s2][0][lane] = make_float4(hA[0], hA[1], hA[2], hA[3]);
            R.ab[s2][1][lane] = make_float4(hB[0], hB[1], hB[2], hB[3]);
            const float ofA[4] = {oA.x, oA.y, oA.z, oA.w}, ofB[4] = {oB.x, oB.y, oB.z, oB.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                uA[j] = __fsub_rn(__fadd_rn(uA[j], hA[j]), ofA[j]);
                uB[j] = __fsub_rn(__fadd_rn(uB[j], hB[j]), ofB[j]);
            }
            if (((r - GR) & 15) == 4) {             // anchor: first-round rows c1-8..c1 afresh
#pragma unroll
                for (int j = 0; j < 4; j++) uA[j] = uB[j] = 0.f;
#pragma unroll
                for (int k = 1; k <= GS_RING; k++) {
                    const int sl = s2 + k < GS_RING ? s2 + k : s2 + k - GS_RING;
                    const float4 a4 = R.ab[sl][0][lane], b4 = R.ab[sl][1][lane];
                    const float ai[4] = {a4.x, a4.y, a4.z, a4.w}, bi[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        uA[j] = __fadd_rn(uA[j], ai[j]);
                        uB[j] = __fadd_rn(uB[j], bi[j]);
                    }
                }
            }
            s2 = s2 == GS_RING - 1 ? 0 : s2 + 1;
        }
        if (r < ys + 2 * GR) return;                // first-round rows c1-8..c1 not all in yet
        if (lane < 2 || lane >= 30) return;         // halo lanes
        // output row y = r - 8; its I is the oldest row of the first ring (slot s1)
        const int y = r - 2 * GR;
        const float icy = inv_count(y, H);
        const float4 Iy = R.ip[s1][0][lane];
        const float Iv[4] = {Iy.x, Iy.y, Iy.z, Iy.w};
        float dy[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float inv = __fmul_rn(icx[j], icy);
            dy[j] = __fmaf_rn(__fmul_rn(uA[j], inv), Iv[j], __fmul_rn(uB[j], inv));
        }
        put_row<FAST>(p, y, cx, dy, in.ow);
    };

    // two load buffers in turn, so a row's loads are in flight while the
    // previous row is computed (no register copy that would wait on them)
    const int r0 = ys - 2 * GR, r1 = ye + 2 * GR;
    RowLoad<FAST> A, B;
    A.issue(p, r0, cx);
    for (int r = r0; r < r1; r += 2) {
        if (r + 1 < r1) B.issue(p, r + 1, cx);
        step(A, r);
        if (r + 1 >= r1) break;
        if (r + 2 < r1) A.issue(p, r + 2, cx);
        step(B, r + 1);
    }
}

__device__ __forceinline__ bool sweep_fast(const TransferParams& p) {
    return p.src_u8 && !(p.w & 3) && (long long)p.w * p.h < (1LL << 29) &&
           !(reinterpret_cast<uintptr_t>(p.src_u8) & 3) &&
           !(reinterpret_cast<uintptr_t>(p.gray_out) & 15) &&
           !(reinterpret_cast<uintptr_t>(p.out_u8) & 3) && !(reinterpret_cast<uintptr_t>(p.out_f32) & 15);
}

// block (bx, by): strips GS_WARPS*bx .. +GS_WARPS-1 of segment by
__device__ __forceinline__ void guided_body(const TransferParams& p, int bx, int by) {
    __shared__ SweepRing rings[GS_WARPS];
    const int w = threadIdx.x >> 5;
    if (sweep_fast(p)) guided_sweep<true>(p, rings[w], bx * GS_WARPS + w, by);
    else guided_sweep<false>(p, rings[w], bx * GS_WARPS + w, by);
}

// ---- rows per segment, per device (the autotuner may change it)
static std::atomic<int> g_seg_rows[64];

int guided_rows(int dev) {
    const int v = (dev >= 0 && dev < 64) ? g_seg_rows[dev].load() : 0;
    return v > 0 ? v : GS_ROWS_DEFAULT;
}

bool guided_set_rows(int dev, int rows) {
    if (dev < 0 || dev >= 64 || rows < 16 || rows > 4096 || (rows & 15)) return false;
    g_seg_rows[dev].store(rows);
    return true;
}

static int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
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
            v = __fadd_rn(pl_ld(p.gray_out, pi, p.h16), -I);
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

__global__ void __launch_bounds__(GS_THREADS) k_guided_transfer(SpArgs args) {
    guided_body(args.p, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(SP_THREADS) k_gauss_transfer(SpArgs args) {
    gauss_body(args.p, blockIdx.x, blockIdx.y);
}
// batched: task = one stream (edge-aware and Gaussian streams in separate launches)
__global__ void __launch_bounds__(GS_THREADS)
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
    // the sweep's rings are static shared memory; prefer shared memory over L1
    cudaError_t e = cudaFuncSetAttribute(k_guided_transfer, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guided_transfer_multi, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    return e;
}

// guided filter: blocks of GS_WARPS strips x one segment of seg_rows rows
// (seg_rows filled from the device's setting when 0); Gaussian: 32x32 tiles
unsigned transfer_grid(TransferParams& p, unsigned& gx, unsigned& gy) {
    if (p.edge_aware) {
        if (p.seg_rows <= 0) p.seg_rows = guided_rows(current_device());
        const int strips = (p.w + GS_OUT - 1) / GS_OUT;
        gx = (unsigned)((strips + GS_WARPS - 1) / GS_WARPS);
        gy = (unsigned)((p.h + p.seg_rows - 1) / p.seg_rows);
    } else {
        gx = (unsigned)((p.w + TS - 1) / TS);
        gy = (unsigned)((p.h + TS - 1) / TS);
    }
    return gx * gy;
}

cudaError_t launch_transfer_multi(int edge_aware, const TransferParams* d_params, const int* d_map,
                                  unsigned blocks, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    if (edge_aware)
        k_guided_transfer_multi<<<blocks, GS_THREADS, 0, st>>>(d_params, d_map);
    else
        k_gauss_transfer_multi<<<blocks, SP_THREADS, 0, st>>>(d_params, d_map);
    return cudaGetLastError();
}

// One stream's frame, waited for by the per-stream path, so latency counts:
// segments short enough that the frame's strips x segments give about eight
// warps per SM (multiples of 16 rows, at most the batched setting).  The
// output is the same whatever the segment height.
cudaError_t launch_transfer(const TransferParams& p0, cudaStream_t st) {
    SpArgs a{p0};
    if (a.p.edge_aware && a.p.seg_rows <= 0) {
        const long long strips = (a.p.w + GS_OUT - 1) / GS_OUT;
        const long long want = 148LL * 8;
        long long rows = (strips * a.p.h + want - 1) / want;
        rows = (rows + 15) / 16 * 16;
        a.p.seg_rows = (int)std::min<long long>(std::max<long long>(rows, 16), guided_rows(current_device()));
    }
    unsigned gx, gy;
    transfer_grid(a.p, gx, gy);
    dim3 grid(gx, gy);
    if (a.p.edge_aware) k_guided_transfer<<<grid, GS_THREADS, 0, st>>>(a);
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

// ---- the autotuner's trial of the segment height: one launch of the sweep
// over a 3840 x 8640 RGB24 frame (four 2160-row frames' worth of strips and
// segments, about the batched tick's warp count at 128 rows), each candidate
// timed over five launches after one warm-up; the fastest is kept.  Outputs
// do not depend on the choice.
cudaError_t guided_autotune(int dev, const int* cand, int nc, float* ms, int* chosen) {
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    const int W = 3840, H = 4 * 2160;
    const size_t P = (size_t)W * H;
    uint8_t *in = nullptr, *out = nullptr;
    float* gray = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    auto done = [&](cudaError_t r) {
        if (in) cudaFree(in);
        if (out) cudaFree(out);
        if (gray) cudaFree(gray);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
        return r;
    };
    if ((e = cudaMalloc(&in, 3 * P)) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&out, 3 * P)) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&gray, P * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(in, 0x5a, 3 * P)) != cudaSuccess) return done(e);
    if ((e = cudaMemset(gray, 0, P * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return done(e);
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) return done(e);
    if ((e = spatial_prepare_device()) != cudaSuccess) return done(e);
    int best = guided_rows(dev);
    float best_ms = 1e30f;
    for (int k = 0; k < nc; k++) {
        SpArgs a{};
        a.p.w = W;
        a.p.h = H;
        a.p.vec_end = (long long)P;
        a.p.src_u8 = in;
        a.p.gray_out = gray;
        a.p.out_u8 = out;
        a.p.edge_aware = 1;
        a.p.seg_rows = cand[k];
        unsigned gx, gy;
        transfer_grid(a.p, gx, gy);
        for (int rep = 0; rep < 6; rep++) {
            if (rep == 1 && (e = cudaEventRecord(e0, st)) != cudaSuccess) return done(e);
            k_guided_transfer<<<dim3(gx, gy), GS_THREADS, 0, st>>>(a);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return done(e);
        if ((e = cudaEventRecord(e1, st)) != cudaSuccess) return done(e);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return done(e);
        float t = 0.f;
        if ((e = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) return done(e);
        ms[k] = t / 5.f;
        if (ms[k] < best_ms) {
            best_ms = ms[k];
            best = cand[k];
        }
    }
    guided_set_rows(dev, best);
    *chosen = best;
    return done(cudaSuccess);
}

}  // namespace wema
