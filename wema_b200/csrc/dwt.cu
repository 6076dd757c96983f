// dwt.cu - 2D CDF 9/7 lifting DWT, forward and inverse, one fused kernel per
// pyramid level.
//
// A CTA owns a tile of TP x TP subband pairs (TP = 27) and stages a 64 x 64
// sample region - the tile's 54 samples plus a 4-sample halo before and a
// 6-sample halo after, clipped at the image - in shared memory, one plane per
// channel it handles (level 0 of a colour frame: all three, so each RGB
// pixel is converted once; otherwise one channel per CTA).  Lifting runs in
// registers: a warp takes one line of the region, lane k holding the sample
// pair (2k, 2k+1), and each of the four lifting steps is one warp shuffle for
// the neighbour plus one FMA.  Rows first, then the tile's columns (forward);
// columns over the whole region, then the tile's rows (inverse).
//
// Sample and pair indices are 32-bit: the runtime caps frames at 2^28 pixels.
//
// Shared layout: even and odd samples are stored apart in both directions -
// sample (y, x) at row (y & 1) * 32 + (y >> 1), column (x & 1) * 48 + (x >> 1)
// of a plane with an odd row stride - so a warp's row or column access, its
// staging of 32 consecutive pixels and its quadrant reads and writes all hit
// 32 distinct banks, and the four subband quadrants are contiguous blocks.
//
// Every output depends only on samples within 4 of it, so with the halo each
// tile is independent: at the image border the reference's whole-sample
// mirror applies (dwt.c:63-98, 126-160); at a tile border the halo is real
// data, and the garbage that the staged segment's own ends produce moves
// inward by at most two lanes, all inside the halo.  Arithmetic is the
// reference's: x = fma(left + right, c, x), scalings as separate multiplies
// (dwt.c:45-170 as GCC -Ofast evaluates it), so coefficients are bit-exact.
#include <atomic>
#include <type_traits>

#include "cascade.cuh"
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

namespace wema {

constexpr int TP = 27;                 // subband pairs per tile side
constexpr int SEG = 64;                // staged samples per line (32 lanes x 2)
constexpr int HALO_L = 4;
constexpr int ODD_COL = 48;            // first column of the odd samples
constexpr int RS = 81;                 // plane row stride (odd, >= ODD_COL + 32)
constexpr int PLANE = SEG * RS;        // floats per staged plane
constexpr int DWT_THREADS = 256;
constexpr int NWARP = DWT_THREADS / 32;
constexpr unsigned FULL = 0xffffffffu;

// first staged sample of the tile starting at pair p0 (even)
__device__ __forceinline__ int seg_start(int p0) { return p0 == 0 ? 0 : 2 * p0 - HALO_L; }
__device__ __forceinline__ int prow(int y) { return (y & 1) * 32 + (y >> 1); }
__device__ __forceinline__ int pcol(int x) { return (x & 1) * ODD_COL + (x >> 1); }

// Forward lifting of one line: lane holds samples s = g0 + 2*lane (even) and
// s + 1 of a line of n samples.  EDGE false: every lane's neighbours lie in
// the line (1 <= g0 and g0 + 64 < n), so the border mirror's selects go.
template <bool EDGE>
__device__ __forceinline__ void lift_fwd(float& e, float& o, int s, int n) {
    const bool r_ok = !EDGE || s + 2 < n;     // predict: right even neighbour s+2
    const bool l_ok = !EDGE || s >= 1;        // update: left odd neighbour s-1
    const bool ro_ok = !EDGE || s + 1 < n;    // update: right odd neighbour s+1
    float t;
#define WEMA_PREDICT(C)                                    \
    t = __shfl_down_sync(FULL, e, 1);                       \
    o = __fmaf_rn(__fadd_rn(e, r_ok ? t : e), C, o);
#define WEMA_UPDATE(C)                                     \
    t = __shfl_up_sync(FULL, o, 1);                         \
    e = __fmaf_rn(__fadd_rn(l_ok ? t : o, ro_ok ? o : t), C, e);
    WEMA_PREDICT(kAlpha)
    WEMA_UPDATE(kBeta)
    WEMA_PREDICT(kGamma)
    WEMA_UPDATE(kDelta)
    e = __fmul_rn(e, kKInv);
    o = __fmul_rn(o, kK);
}

// Inverse lifting of one line (dwt.c:109-170): unscale, then the steps in
// reverse order with negated constants.
template <bool EDGE>
__device__ __forceinline__ void lift_inv(float& e, float& o, int s, int n) {
    const bool r_ok = !EDGE || s + 2 < n;
    const bool l_ok = !EDGE || s >= 1;
    const bool ro_ok = !EDGE || s + 1 < n;
    float t;
    e = __fmul_rn(e, kK);
    o = __fmul_rn(o, kKInv);
    WEMA_UPDATE(-kDelta)
    WEMA_PREDICT(-kGamma)
    WEMA_UPDATE(-kBeta)
    WEMA_PREDICT(-kAlpha)
#undef WEMA_PREDICT
#undef WEMA_UPDATE
}

// LPW lines of one plane at a time (2, 4 or 8: a tuning choice, the result
// is the same): their lifting chains are independent, so the warp
// interleaves them.  b[u] is line u's base (a valid line even when
// act[u] is false - then nothing is stored); ei / oi address this lane's even
// and odd sample, s is its even sample's global index, n the line length, lim
// the staged length.  s0 is lane 0's s: a segment away from both ends of
// the line (s0 >= 1, s0 + 64 < n) lifts without the border selects.
template <bool FWD, int LPW>
__device__ __forceinline__ void liftN(float* const (&b)[LPW], const bool (&act)[LPW], int ei, int oi,
                                      int s0, int n, int lim, int lane) {
    const int s = s0 + 2 * lane;
    float e[LPW], o[LPW];
#pragma unroll
    for (int u = 0; u < LPW; u++) {
        e[u] = b[u][ei];
        o[u] = b[u][oi];
    }
    if (s0 >= 1 && s0 + SEG < n) {
#pragma unroll
        for (int u = 0; u < LPW; u++) {
            if (FWD) lift_fwd<false>(e[u], o[u], s, n);
            else lift_inv<false>(e[u], o[u], s, n);
        }
    } else {
#pragma unroll
        for (int u = 0; u < LPW; u++) {
            if (FWD) lift_fwd<true>(e[u], o[u], s, n);
            else lift_inv<true>(e[u], o[u], s, n);
        }
    }
#pragma unroll
    for (int u = 0; u < LPW; u++) {
        if (!act[u]) continue;
        if (2 * lane < lim) b[u][ei] = e[u];
        if (2 * lane + 1 < lim) b[u][oi] = o[u];
    }
}

// The temporal filter's step (cascade.cuh) on the three coefficients of one
// position of a level, LH / HH / HL (slots 0-2, unique offsets b*n + o), as
// the forward transform writes them: the filter reads the coefficient as
// stored (FP16-rounded in the planes_fp16 variant), so the deltas equal
// those of the separate filter kernel bit for bit.  All state loads first.
// all_simd: no coefficient of the CTA's tile takes the scalar-tail form
// (uniform over the CTA), so the per-coefficient test and select drop out.
__device__ __forceinline__ void temporal_step3(const FwdLevelParams& p, int ch, void* st, int o, int n,
                                               const float (&v)[3], bool h, bool all_simd) {
    float x[3];
#pragma unroll
    for (int b = 0; b < 3; b++) x[b] = h ? __half2float(__float2half_rn(v[b])) : v[b];
    float* dl = p.iir_delta[ch];
    if (p.iir_fp64) {
        double2* s2 = static_cast<double2*>(st);
        double2 hp[3], lp[3];
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const int u = b * n + o;
            hp[b] = __ldcs(s2 + 2 * (long long)u);
            lp[b] = __ldcs(s2 + 2 * (long long)u + 1);
        }
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const int u = b * n + o;
            pl_st(dl, u, cascade64(p.iir_c, hp[b], lp[b], x[b]), h);
            __stcs(s2 + 2 * (long long)u, hp[b]);
            __stcs(s2 + 2 * (long long)u + 1, lp[b]);
        }
    } else {
        float4* s4 = static_cast<float4*>(st);
        float4 sv[3];
#pragma unroll
        for (int b = 0; b < 3; b++) sv[b] = __ldcs(s4 + (b * n + o));   // touched once: evict first
        if (all_simd) {   // the whole tile before the scalar-tail positions (uniform)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int u = b * n + o;
                pl_st(dl, u, cascade(p.iir_c, sv[b], x[b], false), h);
                __stcs(s4 + u, sv[b]);
            }
        } else {
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int u = b * n + o;
                const bool tail = p.iir_off6 + u >= p.iir_simd_end;
                pl_st(dl, u, cascade(p.iir_c, sv[b], x[b], tail), h);
                __stcs(s4 + u, sv[b]);
            }
        }
    }
}

// Bulk L2 prefetch (cp.async.bulk.prefetch.L2) of the IIR state of a tile's
// positions: per band, each of the tile's rows is one contiguous run of
// min(TP, sw - px0) positions (16 B each, or 32 B with the FP64 state), so
// the sizes and addresses are multiples of 16 bytes.  One thread per run.
__device__ __forceinline__ void prefetch_state_rows(const FwdLevelParams& p, int ch, int px0, int py0) {
    const int ni = min(TP, p.sw - px0), nj = min(TP, p.sh - py0);
    const int k = threadIdx.x;
    if (ni <= 0 || k >= 3 * nj) return;
    const int b = k / nj, jj = k - b * nj;
    const long long u = (long long)b * p.n + (long long)(py0 + jj) * p.sw + px0;
    const int esz = p.iir_fp64 ? 32 : 16;
    const char* a = static_cast<const char*>(p.iir_state[ch]) + u * esz;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(ni * esz) : "memory");
}

// ----------------------------------------------------------------- forward
// C == 3: level 0 of a colour frame, all channels in one CTA, grid (tx, ty, 1).
// C == 1: channel blockIdx.z (planes in), or the luma of an RGB frame.
// H16: the planes_fp16 variant's FP16 coefficient planes (p.h16), a
// compile-time constant so the FP32 path carries no FP16 selects
// FULL: the staged region is a whole 64 x 64 inside the level, as in the
// inverse (inv_full), so the tile is a whole 27 x 27 pairs with every odd
// sample present and the bounds tests fold away.
__device__ __forceinline__ bool fwd_full(const FwdLevelParams& p, int bx, int by) {
    return p.iw - seg_start(bx * TP) >= SEG && p.ih - seg_start(by * TP) >= SEG;
}
template <int C, int MODE, int LPW, bool H16, bool FULL>
__device__ __forceinline__ void dwt_fwd_body(const FwdLevelParams& p, int bx, int by, int bz) {
    extern __shared__ __align__(16) float dyn[];
    float* planes = dyn;                                   // [C][PLANE]
    const int ch0 = (C == 1 && MODE == kSrcPlanes) ? bz : 0;
    const int iw = p.iw, ih = p.ih, sw = p.sw, sh = p.sh;
    const int px0 = bx * TP, py0 = by * TP;
    const int rx0 = seg_start(px0), ry0 = seg_start(py0);
    const int RW = FULL ? SEG : min(SEG, iw - rx0), RH = FULL ? SEG : min(SEG, ih - ry0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // the IIR state rows this tile's write-out will update: bulk prefetches
    // into L2 now, so the epilogue's state loads do not wait on DRAM
    if (C == 1 && p.iir_state[ch0]) prefetch_state_rows(p, ch0, px0, py0);

    // ---- staging: one warp per region row
    // every load of the warp's rows is issued before any is used
    constexpr int RPW = SEG / NWARP;   // region rows per warp
    if (MODE == kSrcPlanes) {
        float v[RPW][2];
#pragma unroll
        for (int r = 0; r < RPW; r++) {
            const int ly = warp + r * NWARP;
            const int row0 = (ry0 + ly) * iw + rx0;
            v[r][0] = (ly < RH && lane < RW) ? __ldg(p.src_planes[ch0] + row0 + lane) : 0.0f;
            v[r][1] = (ly < RH && lane + 32 < RW) ? __ldg(p.src_planes[ch0] + row0 + lane + 32) : 0.0f;
        }
#pragma unroll
        for (int r = 0; r < RPW; r++) {
            const int ly = warp + r * NWARP;
            if (ly >= RH) continue;
            float* dst = planes + prow(ly) * RS;
            if (lane < RW) dst[pcol(lane)] = v[r][0];
            if (lane + 32 < RW) dst[pcol(lane + 32)] = v[r][1];
        }
    } else {
        float rgb[RPW][2][3];
        // lane k holds pixels 2k and 2k + 1 of each of its rows (rgb[r][0], [1])
        if (MODE == kSrcRgbU8) {
            // the lane's 6 bytes at byte off + 6k of the row: the (at most 3)
            // aligned 32-bit words holding them, loaded directly (neighbouring
            // lanes share words through L1; an aligned word that holds a byte of
            // the frame is mapped memory, words past the row's last are not read)
            uint32_t wv[RPW][3];
            int sh[RPW];
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                const int ly = warp + r * NWARP;
                const uintptr_t a0 = reinterpret_cast<uintptr_t>(
                    p.src_u8 + 3 * ((ry0 + min(ly, RH - 1)) * iw + rx0));
                const uint32_t* w0 = reinterpret_cast<const uint32_t*>(a0 & ~(uintptr_t)3);
                const int off = (int)(a0 & 3);
                const int nw = (off + 3 * RW + 3) >> 2;
                const int wb = (off + 6 * lane) >> 2;
                sh[r] = 8 * ((off + 6 * lane) & 3);
                const bool row = ly < RH && 2 * lane < RW;
#pragma unroll
                for (int k = 0; k < 3; k++) wv[r][k] = (row && wb + k < nw) ? __ldg(w0 + wb + k) : 0u;
            }
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                const uint32_t x0 = __funnelshift_r(wv[r][0], wv[r][1], sh[r]);   // bytes 0-3
                const uint32_t x1 = __funnelshift_r(wv[r][1], wv[r][2], sh[r]);   // bytes 4-7
                rgb[r][0][0] = byte_of(x0, 0);      // fl(byte / 255)
                rgb[r][0][1] = byte_of(x0, 1);
                rgb[r][0][2] = byte_of(x0, 2);
                rgb[r][1][0] = byte_of(x0, 3);
                rgb[r][1][1] = byte_of(x1, 0);
                rgb[r][1][2] = byte_of(x1, 1);
            }
        } else {
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                const int ly = warp + r * NWARP;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int lx = 2 * lane + h;
                    const bool ok = ly < RH && lx < RW;
                    const float* q = p.src_f32 + 3 * ((ry0 + (ok ? ly : 0)) * iw + rx0 + (ok ? lx : 0));
                    rgb[r][h][0] = q[0];
                    rgb[r][h][1] = q[1];
                    rgb[r][h][2] = q[2];
                }
            }
        }
        float* pout[C];
#pragma unroll
        for (int cc = 0; cc < C; cc++) pout[cc] = p.plane_out[cc];
        const long long vec_end = p.vec_end;
        // ALL: the whole staged region lies in the vector body (every tile but
        // the frame's last ones), so no pixel needs the epilogue's form
        auto convert = [&](auto all) {
            constexpr bool ALL = decltype(all)::value;
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                const int ly = warp + r * NWARP;
                if (ly >= RH) continue;
                const int rowpix = (ry0 + ly) * iw + rx0;
                const bool rowvec = ALL || rowpix + RW <= vec_end;   // the whole staged row in the vector body
                float* dst = planes + prow(ly) * RS;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int lx = 2 * lane + h;
                    if (lx >= RW) continue;
                    const int pi = rowpix + lx;
                    const bool vec = rowvec || pi < vec_end;
                    const float rr = rgb[r][h][0], gg = rgb[r][h][1], bb = rgb[r][h][2];
                    float out[3];
                    if (C == 1) {
                        out[0] = (ALL || vec) ? luma_vec(rr, gg, bb) : luma_tail(rr, gg, bb);
                    } else if (ALL || vec) {
                        ycbcr_vec(rr, gg, bb, out[0], out[1], out[2]);
                    } else {
                        ycbcr_tail(rr, gg, bb, out[0], out[1], out[2]);
                    }
#pragma unroll
                    for (int cc = 0; cc < C; cc++) {
                        dst[cc * PLANE + pcol(lx)] = out[cc];
                        if (pout[cc]) pout[cc][pi] = out[cc];
                    }
                }
            }
        };
        if ((long long)(ry0 + RH - 1) * iw + rx0 + RW <= vec_end) convert(std::true_type{});
        else convert(std::false_type{});
    }
    __syncthreads();

    if (iw >= 2) {   // rows: every staged row of every plane
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int l0 = warp; l0 < RH; l0 += LPW * NWARP) {
                float* b[LPW];
                bool act[LPW];
#pragma unroll
                for (int u = 0; u < LPW; u++) {
                    const int ly = l0 + u * NWARP;
                    act[u] = ly < RH;
                    b[u] = planes + cc * PLANE + prow(min(ly, RH - 1)) * RS;
                }
                liftN<true, LPW>(b, act, lane, ODD_COL + lane, rx0, iw, RW, lane);
            }
        __syncthreads();
    }
    const int cx0 = 2 * px0 - rx0, cx1 = min(2 * (px0 + TP), iw) - rx0;
    if (ih >= 2) {   // columns: the tile's own
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int l0 = cx0 + warp; l0 < cx1; l0 += LPW * NWARP) {
                float* b[LPW];
                bool act[LPW];
#pragma unroll
                for (int u = 0; u < LPW; u++) {
                    const int lx = l0 + u * NWARP;
                    act[u] = lx < cx1;
                    b[u] = planes + cc * PLANE + pcol(min(lx, cx1 - 1));
                }
                liftN<true, LPW>(b, act, lane * RS, (32 + lane) * RS, ry0, ih, RH, lane);
            }
        __syncthreads();
    }

    // quadrants: LL (even,even), HL (odd x), LH (odd y), HH; stale entries of
    // odd-sized levels take the previous level's value at the same index
    const int ni = FULL ? TP : min(TP, sw - px0), nj = FULL ? TP : min(TP, sh - py0);
    const int qx0 = px0 - (rx0 >> 1), qy0 = py0 - (ry0 >> 1);   // tile's first pair in the region
    const int i = px0 + lane;
    const bool hx = FULL || 2 * i + 1 < iw;
    const int n = (int)p.n, pn = (int)p.prev_n;
    // every coefficient of the tile lies before the scalar-tail positions of
    // the 6-slot array (all but the last tiles of a frame's last level)
    const bool all_simd = p.iir_off6 + 2 * p.n + (long long)(py0 + nj - 1) * sw + px0 + ni - 1 < p.iir_simd_end;
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
        const int ch = ch0 + cc;
        const float* pl = planes + cc * PLANE + qx0 + lane;
        float* ll = p.ll_out[ch];
        float* bands = p.coef[ch];
        const float* prev = p.prev[ch];
        void* const st = p.iir_state[ch];
        for (int jj = warp; jj < nj; jj += NWARP) {
            if (lane >= ni) continue;
            const int j = py0 + jj, ry = qy0 + jj;
            const int o = j * sw + i;
            const bool hy = FULL || 2 * j + 1 < ih;
            constexpr bool h = H16;
            float v[3];                                                                         // LH, HH, HL
            v[0] = hy ? pl[(32 + ry) * RS] : (prev ? pl_ld(prev, o, h) : 0.0f);
            v[1] = (hx && hy) ? pl[(32 + ry) * RS + ODD_COL] : (prev ? pl_ld(prev, pn + o, h) : 0.0f);
            v[2] = hx ? pl[ry * RS + ODD_COL] : (prev ? pl_ld(prev, 2 * pn + o, h) : 0.0f);
            ll[o] = pl[ry * RS];
#pragma unroll
            for (int b = 0; b < 3; b++) pl_st(bands, b * n + o, v[b], h);
            if (st) temporal_step3(p, ch, st, o, n, v, h, all_simd);
        }
    }
}

// ----------------------------------------------------------------- inverse
// C == 1: grid (tiles_x, tiles_y, channels), planes out.
// C == 3: one CTA per tile does all three channels (YCbCr -> RGB at level 0).
// H16: FP16 coefficient / delta planes and (p.out16) FP16 output planes,
// a compile-time constant as in the forward body.  FULL: the staged region is
// a whole 64 x 64 inside the level (every tile but those at the far edges),
// so its extent is a constant and the bounds tests fold away.
__device__ __forceinline__ bool inv_full(const InvLevelParams& p, int bx, int by) {
    return p.ow - seg_start(bx * TP) >= SEG && p.oh - seg_start(by * TP) >= SEG;
}
template <int C, int OUT, int LPW, bool H16, bool FULL>
__device__ __forceinline__ void dwt_inv_body(const InvLevelParams& p, int bx, int by, int bz) {
    extern __shared__ __align__(16) float dyn[];
    float* planes = dyn;   // [C][PLANE]
    const int ow = p.ow, oh = p.oh, sw = p.sw, sh = p.sh;
    const int px0 = bx * TP, py0 = by * TP;
    const int rx0 = seg_start(px0), ry0 = seg_start(py0);
    const int RW = FULL ? SEG : min(SEG, ow - rx0), RH = FULL ? SEG : min(SEG, oh - ry0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = (C == 1) ? bz : 0;
    const int gx0 = rx0 >> 1, gy0 = ry0 >> 1;   // region's first pair

    // ---- staging: quadrant q (0 LL, 1 HL, 2 LH, 3 HH) of a plane is a 32 x 32
    // block of one subband, its rows 32 consecutive pairs; bands are amplified
    // on the way in.  Each warp takes rows warp, warp + 8, ... of every block,
    // all of its loads before any store.
    const int n = (int)p.n;
    const int o0 = gy0 * sw + gx0 + lane;
    float xv[C][4][4], dv[C][3][4];   // every load of the warp's rows first
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
        const int ch = c0 + cc;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int boff = q == 1 ? 2 * n : (q == 2 ? 0 : n);   // HL 2, LH 0, HH 1
            const float* src = q == 0 ? p.ll[ch] : plane_at(p.coef[ch], boff, H16);
            const float* dsrc = plane_at(p.delta[ch], boff, H16);
            const bool okx = 2 * lane + (q & 1) < RW;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int qy = warp + NWARP * u;
                const bool ok = okx && 2 * qy + (q >> 1) < RH;
                const int o = o0 + qy * sw;
                xv[cc][q][u] = ok ? pl_ld(src, o, q != 0 && H16) : 0.0f;
                if (q != 0) dv[cc][q - 1][u] = ok ? pl_ld(dsrc, o, H16) : 0.0f;
            }
        }
    }
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
        const int ch = c0 + cc;
        const float thr = p.thr[ch], al = p.alpha[ch];
        float* pl = planes + cc * PLANE + lane;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int xo = q & 1, yo = q >> 1;
            const bool okx = 2 * lane + xo < RW;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int qy = warp + NWARP * u;
                if (!(okx && 2 * qy + yo < RH)) continue;
                float x = xv[cc][q][u];
                if (q != 0 && fabsf(x) > thr) x = __fmaf_rn(dv[cc][q - 1][u], al, x);
                pl[(yo * 32 + qy) * RS + xo * ODD_COL] = x;
            }
        }
    }
    (void)sh;
    __syncthreads();
    if (oh >= 2) {   // columns over the whole staged region
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int l0 = warp; l0 < RW; l0 += LPW * NWARP) {
                float* b[LPW];
                bool act[LPW];
#pragma unroll
                for (int u = 0; u < LPW; u++) {
                    const int lx = l0 + u * NWARP;
                    act[u] = lx < RW;
                    b[u] = planes + cc * PLANE + pcol(min(lx, RW - 1));
                }
                liftN<false, LPW>(b, act, lane * RS, (32 + lane) * RS, ry0, oh, RH, lane);
            }
        __syncthreads();
    }
    const int ty0 = 2 * py0 - ry0, ty1 = FULL ? ty0 + 2 * TP : min(2 * (py0 + TP), oh) - ry0;
    const int tx0 = 2 * px0 - rx0, tx1 = FULL ? tx0 + 2 * TP : min(2 * (px0 + TP), ow) - rx0;
    if (ow >= 2) {   // rows of the tile
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int l0 = ty0 + warp; l0 < ty1; l0 += LPW * NWARP) {
                float* b[LPW];
                bool act[LPW];
#pragma unroll
                for (int u = 0; u < LPW; u++) {
                    const int ly = l0 + u * NWARP;
                    act[u] = ly < ty1;
                    b[u] = planes + cc * PLANE + prow(min(ly, ty1 - 1)) * RS;
                }
                liftN<false, LPW>(b, act, lane, ODD_COL + lane, rx0, ow, RW, lane);
            }
        __syncthreads();
    }
    // ---- output: one warp per tile row, lanes along x
    const bool out16 = H16 && p.out16;
    if (OUT == kOutPlanes) {
        // two adjacent pixels per lane: the even one from the row's even half in
        // shared memory, the odd one ODD_COL further (tx0 is even), one index
        // computation for both and, on an even pixel index, one 8-byte store
        for (int ly = ty0 + warp; ly < ty1; ly += NWARP) {
            const int lx = tx0 + 2 * lane;
            if (lx >= tx1) continue;
            const int pi = (ry0 + ly) * ow + rx0 + lx;
            const int ie = prow(ly) * RS + (lx >> 1);
            const bool two = lx + 1 < tx1;
#pragma unroll
            for (int cc = 0; cc < C; cc++) {
                float* o = p.out_planes[c0 + cc];
                const float ve = planes[cc * PLANE + ie];
                const float vo = two ? planes[cc * PLANE + ie + ODD_COL] : 0.0f;
                if (!out16 && two && !(pi & 1)) {
                    *reinterpret_cast<float2*>(o + pi) = make_float2(ve, vo);
                } else {
                    pl_st(o, pi, ve, out16);
                    if (two) pl_st(o, pi + 1, vo, out16);
                }
            }
        }
    } else {   // RGB out (colour level 0)
        for (int ly = ty0 + warp; ly < ty1; ly += NWARP) {
            const int rowpix = (ry0 + ly) * ow + rx0;
            const int pr = prow(ly) * RS;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int lx = tx0 + lane + 32 * h;
                if (lx >= tx1) continue;
                const int pi = rowpix + lx;
                const int idx = pr + pcol(lx);
                const float y = planes[idx];
                const float cb = planes[(C > 1 ? PLANE : 0) + idx];
                const float cr = planes[(C > 2 ? 2 * PLANE : 0) + idx];
                if (p.out_planes[0]) {
                    pl_st(p.out_planes[0], pi, y, out16);
                    pl_st(p.out_planes[1], pi, cb, out16);
                    pl_st(p.out_planes[2], pi, cr, out16);
                }
                float r, g, b;
                ycbcr_to_rgb(y, cb, cr, r, g, b);
                if (p.out_u8) {
                    uint8_t* d = p.out_u8 + 3 * pi;
                    d[0] = quant_u8(r);
                    d[1] = quant_u8(g);
                    d[2] = quant_u8(b);
                }
                if (p.out_f32) {
                    float* d = p.out_f32 + 3 * pi;
                    d[0] = r;
                    d[1] = g;
                    d[2] = b;
                }
            }
        }
    }
}

// ------------------------------------------------------------- wrappers
// one stream per launch, and the batched form (task = stream; params in device
// memory, one entry per task).  The batched luma kernels also come in tuning
// variants: MINB CTAs per SM asked of the register allocator (1: the
// compiler's choice, 3 or 4) and
// LPW lines per warp in flight (2, 4 or 8); every variant computes the same
// coefficients, bit for bit.
constexpr int LPW_DEF = 4;
// Plane type (FP32, or the planes_fp16 variant's FP16): one stream's kernel
// is compiled for its type (H16, chosen at launch); a batched launch whose
// tasks are all FP32 takes the FP32-only kernel, one with FP16-plane tasks
// (ANY16) the kernel holding both bodies, chosen per CTA.  A kernel holding
// both is allocated registers for both, which slowed the FP32 colour path.
template <int C, int MODE, bool H16>
__global__ void __launch_bounds__(DWT_THREADS, 3) k_dwt_fwd(FwdLevelParams p) {
    if (!H16 && fwd_full(p, blockIdx.x, blockIdx.y))
        dwt_fwd_body<C, MODE, LPW_DEF, false, true>(p, blockIdx.x, blockIdx.y, blockIdx.z);
    else dwt_fwd_body<C, MODE, LPW_DEF, H16, false>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
// A batched one-channel CTA works on channel z of its task: the task's
// parameters copied into registers with that channel's fields at index 0, the
// body run as channel 0, so every array index in it is a constant (a copy
// indexed by a run-time channel goes to the stack).  Levels 1-3 forward:
// spills about 108 -> 60 bytes, 0.2445 -> 0.239 ms per tick; inverse levels
// 0.119 -> 0.116 and level 0 0.276 -> 0.272 ms; bit-identical.
__device__ __forceinline__ FwdLevelParams fwd_chan(const FwdLevelParams& g, int z) {
    FwdLevelParams q = g;
    q.src_planes[0] = g.src_planes[z];
    q.coef[0] = g.coef[z];
    q.prev[0] = g.prev[z];
    q.ll_out[0] = g.ll_out[z];
    q.iir_state[0] = g.iir_state[z];
    q.iir_delta[0] = g.iir_delta[z];
    return q;
}
__device__ __forceinline__ InvLevelParams inv_chan(const InvLevelParams& g, int z) {
    InvLevelParams q = g;
    q.ll[0] = g.ll[z];
    q.coef[0] = g.coef[z];
    q.delta[0] = g.delta[z];
    q.thr = g.thr + z;
    q.alpha[0] = g.alpha[z];
    q.out_planes[0] = g.out_planes[z];
    return q;
}
template <int C, int MODE, int LPW, bool ANY16>
__device__ __forceinline__ void dwt_fwd_task(const FwdLevelParams& p, const TaskBlock& t) {
    if (ANY16 && p.h16) dwt_fwd_body<C, MODE, LPW, true, false>(p, t.x, t.y, t.z);
    else if (fwd_full(p, t.x, t.y)) dwt_fwd_body<C, MODE, LPW, false, true>(p, t.x, t.y, t.z);
    else dwt_fwd_body<C, MODE, LPW, false, false>(p, t.x, t.y, t.z);
}
template <int C, int MODE, int MINB, int LPW, bool ANY16>
__global__ void __launch_bounds__(DWT_THREADS, MINB)
    k_dwt_fwd_multi(const FwdLevelParams* __restrict__ ps, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    if constexpr (MODE == kSrcRgbU8) {
        // level 0 from RGB24: the task's parameters copied to registers.  Read through a
        // reference into the table, a field is loaded again after stores that
        // may alias the table as far as the compiler knows; the copy cut the
        // spills (about 120 to 28 bytes) and the level's time (0.646 -> 0.615 ms
        // per tick on the 48-stream mix).
        const FwdLevelParams p = ps[t.task];
        dwt_fwd_task<C, MODE, LPW, ANY16>(p, t);
    } else if constexpr (C == 1) {
        const FwdLevelParams p = fwd_chan(ps[t.task], t.z);
        dwt_fwd_task<C, MODE, LPW, ANY16>(p, TaskBlock{t.task, t.x, t.y, 0});
    } else {
        dwt_fwd_task<C, MODE, LPW, ANY16>(ps[t.task], t);
    }
}
// one channel: 4 CTAs per SM (measured in the batched form: 40% faster than the
// compiler's 82-register choice, which leaves 2); colour: 3 CTAs per SM
template <int C, int OUT, bool H16>
__global__ void __launch_bounds__(DWT_THREADS, C == 1 ? 4 : 3) k_dwt_inv(InvLevelParams p) {
    if (!H16 && inv_full(p, blockIdx.x, blockIdx.y))
        dwt_inv_body<C, OUT, LPW_DEF, false, true>(p, blockIdx.x, blockIdx.y, blockIdx.z);
    else dwt_inv_body<C, OUT, LPW_DEF, H16, false>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int C, int OUT, int MINB, int LPW, bool ANY16>
__global__ void __launch_bounds__(DWT_THREADS, MINB)
    k_dwt_inv_multi(const InvLevelParams* __restrict__ ps, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    if constexpr (C == 1) {
        const InvLevelParams p = inv_chan(ps[t.task], t.z);
        if (ANY16 && p.h16) dwt_inv_body<C, OUT, LPW, true, false>(p, t.x, t.y, 0);
        else if (inv_full(p, t.x, t.y)) dwt_inv_body<C, OUT, LPW, false, true>(p, t.x, t.y, 0);
        else dwt_inv_body<C, OUT, LPW, false, false>(p, t.x, t.y, 0);
    } else {
        const InvLevelParams& p = ps[t.task];
        if (ANY16 && p.h16) dwt_inv_body<C, OUT, LPW, true, false>(p, t.x, t.y, t.z);
        else if (inv_full(p, t.x, t.y)) dwt_inv_body<C, OUT, LPW, false, true>(p, t.x, t.y, t.z);
        else dwt_inv_body<C, OUT, LPW, false, false>(p, t.x, t.y, t.z);
    }
}

// ---- tuning of the batched luma kernels, per device: variant index
// v = 3 * minb_index + lpw_index over MINB {1, 3, 4} x LPW {2, 4, 8}
constexpr int kDwtVariants = 9;
static const int kMinb[3] = {1, 3, 4}, kLpw[3] = {2, 4, 8};
static std::atomic<int> g_dwt_var[64][2];     // [device][0 forward, 1 inverse], value + 1

static int dwt_dev_now() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}
int dwt_variant(int dev, int inverse) {
    const int v = (dev >= 0 && dev < 64) ? g_dwt_var[dev][inverse ? 1 : 0].load() : 0;
    // defaults until tuned: the fastest in a 48-stream tick on B200 - 4 CTAs per
    // SM x 4 lines per warp, forward and inverse
    return v > 0 ? v - 1 : 2 * 3 + 1;
}
bool dwt_set_variant(int dev, int inverse, int v) {
    if (dev < 0 || dev >= 64 || v < 0 || v >= kDwtVariants) return false;
    g_dwt_var[dev][inverse ? 1 : 0].store(v + 1);
    return true;
}
void dwt_variant_shape(int v, int* minb, int* lpw) {
    *minb = kMinb[v / 3];
    *lpw = kLpw[v % 3];
}

// ----------------------------------------------------------------- launch

static size_t fwd_smem(int C) { return (size_t)C * PLANE * sizeof(float); }
static size_t inv_smem(int C) { return (size_t)C * PLANE * sizeof(float); }
size_t dwt_smem_bytes(int C) { return fwd_smem(C); }

static unsigned tiles_of(int pairs) { return (unsigned)((pairs + TP - 1) / TP); }

template <class K>
static cudaError_t allow_smem(K k, size_t bytes) {
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// kernels above the 48 KB default; call once per device
cudaError_t dwt_prepare_device() {
    cudaError_t e = allow_smem(k_dwt_inv<3, kOutRgb, false>, inv_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_inv<3, kOutRgb, true>, inv_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd<3, kSrcRgbU8, false>, fwd_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd<3, kSrcRgbU8, true>, fwd_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd<3, kSrcRgbF32, false>, fwd_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd<3, kSrcRgbF32, true>, fwd_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_inv_multi<3, kOutRgb, 3, LPW_DEF, false>, inv_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_inv_multi<3, kOutRgb, 3, LPW_DEF, true>, inv_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd_multi<3, kSrcRgbU8, 3, LPW_DEF, false>, fwd_smem(3));
    if (e == cudaSuccess) e = allow_smem(k_dwt_fwd_multi<3, kSrcRgbU8, 3, LPW_DEF, true>, fwd_smem(3));
    return e;
}

// ---- batched launches: grid = sum of the tasks' grids (map built by the host)
unsigned dwt_fwd_grid(const FwdLevelParams& p, int channels_z, unsigned& gx, unsigned& gy) {
    gx = tiles_of(p.sw);
    gy = tiles_of(p.sh);
    return gx * gy * (unsigned)channels_z;
}
unsigned dwt_inv_grid(const InvLevelParams& p, int channels_z, unsigned& gx, unsigned& gy) {
    gx = tiles_of((p.ow + 1) / 2);
    gy = tiles_of((p.oh + 1) / 2);
    return gx * gy * (unsigned)channels_z;
}

cudaError_t launch_dwt_fwd_multi(int mode, int channels, const FwdLevelParams* d_params,
                                 const int* d_map, unsigned blocks, bool any16, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    if (mode == kSrcRgbU8 && channels == 3) {
        if (any16) k_dwt_fwd_multi<3, kSrcRgbU8, 3, LPW_DEF, true><<<blocks, DWT_THREADS, fwd_smem(3), st>>>(d_params, d_map);
        else k_dwt_fwd_multi<3, kSrcRgbU8, 3, LPW_DEF, false><<<blocks, DWT_THREADS, fwd_smem(3), st>>>(d_params, d_map);
        return cudaGetLastError();
    }
    if ((mode != kSrcPlanes && mode != kSrcRgbU8) || channels != 1) return cudaErrorInvalidValue;
    const int v = dwt_variant(dwt_dev_now(), 0);
    const size_t sm = fwd_smem(1);
#define WEMA_FWD_CASE(I, MB, LP)                                                                        \
    case I:                                                                                             \
        if (mode == kSrcPlanes) {                                                                       \
            if (any16) k_dwt_fwd_multi<1, kSrcPlanes, MB, LP, true><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
            else k_dwt_fwd_multi<1, kSrcPlanes, MB, LP, false><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
        } else {                                                                                        \
            if (any16) k_dwt_fwd_multi<1, kSrcRgbU8, MB, LP, true><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
            else k_dwt_fwd_multi<1, kSrcRgbU8, MB, LP, false><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
        }                                                                                               \
        break;
    switch (v) {
        WEMA_FWD_CASE(0, 1, 2) WEMA_FWD_CASE(1, 1, 4) WEMA_FWD_CASE(2, 1, 8)
        WEMA_FWD_CASE(3, 3, 2) WEMA_FWD_CASE(4, 3, 4) WEMA_FWD_CASE(5, 3, 8)
        WEMA_FWD_CASE(6, 4, 2) WEMA_FWD_CASE(7, 4, 4) WEMA_FWD_CASE(8, 4, 8)
        default: return cudaErrorInvalidValue;
    }
#undef WEMA_FWD_CASE
    return cudaGetLastError();
}

cudaError_t launch_dwt_inv_multi(int channels, int out_mode, const InvLevelParams* d_params,
                                 const int* d_map, unsigned blocks, bool any16, cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    if (out_mode == kOutRgb && channels == 3) {
        if (any16) k_dwt_inv_multi<3, kOutRgb, 3, LPW_DEF, true><<<blocks, DWT_THREADS, inv_smem(3), st>>>(d_params, d_map);
        else k_dwt_inv_multi<3, kOutRgb, 3, LPW_DEF, false><<<blocks, DWT_THREADS, inv_smem(3), st>>>(d_params, d_map);
        return cudaGetLastError();
    }
    if (out_mode != kOutPlanes) return cudaErrorInvalidValue;
    const int v = dwt_variant(dwt_dev_now(), 1);
    const size_t sm = inv_smem(1);
#define WEMA_INV_CASE(I, MB, LP)                                                                        \
    case I:                                                                                             \
        if (any16) k_dwt_inv_multi<1, kOutPlanes, MB, LP, true><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
        else k_dwt_inv_multi<1, kOutPlanes, MB, LP, false><<<blocks, DWT_THREADS, sm, st>>>(d_params, d_map); \
        break;
    switch (v) {
        WEMA_INV_CASE(0, 1, 2) WEMA_INV_CASE(1, 1, 4) WEMA_INV_CASE(2, 1, 8)
        WEMA_INV_CASE(3, 3, 2) WEMA_INV_CASE(4, 3, 4) WEMA_INV_CASE(5, 3, 8)
        WEMA_INV_CASE(6, 4, 2) WEMA_INV_CASE(7, 4, 4) WEMA_INV_CASE(8, 4, 8)
        default: return cudaErrorInvalidValue;
    }
#undef WEMA_INV_CASE
    return cudaGetLastError();
}

cudaError_t launch_dwt_fwd(int mode, int channels, const FwdLevelParams& p, cudaStream_t st) {
    if (channels != 1 && channels != 3) return cudaErrorInvalidValue;
    const unsigned tx = tiles_of(p.sw), ty = tiles_of(p.sh);
    if (mode == kSrcPlanes) {
        if (p.h16) k_dwt_fwd<1, kSrcPlanes, true><<<dim3(tx, ty, channels), DWT_THREADS, fwd_smem(1), st>>>(p);
        else k_dwt_fwd<1, kSrcPlanes, false><<<dim3(tx, ty, channels), DWT_THREADS, fwd_smem(1), st>>>(p);
    } else if (mode == kSrcRgbU8) {
        if (channels == 3 && p.h16) k_dwt_fwd<3, kSrcRgbU8, true><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(3), st>>>(p);
        else if (channels == 3) k_dwt_fwd<3, kSrcRgbU8, false><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(3), st>>>(p);
        else if (p.h16) k_dwt_fwd<1, kSrcRgbU8, true><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(1), st>>>(p);
        else k_dwt_fwd<1, kSrcRgbU8, false><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(1), st>>>(p);
    } else if (mode == kSrcRgbF32) {
        if (channels == 3 && p.h16) k_dwt_fwd<3, kSrcRgbF32, true><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(3), st>>>(p);
        else if (channels == 3) k_dwt_fwd<3, kSrcRgbF32, false><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(3), st>>>(p);
        else if (p.h16) k_dwt_fwd<1, kSrcRgbF32, true><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(1), st>>>(p);
        else k_dwt_fwd<1, kSrcRgbF32, false><<<dim3(tx, ty, 1), DWT_THREADS, fwd_smem(1), st>>>(p);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dwt_inv(int channels, int out_mode, const InvLevelParams& p, cudaStream_t st) {
    const unsigned tx = tiles_of((p.ow + 1) / 2), ty = tiles_of((p.oh + 1) / 2);
    if (out_mode == kOutPlanes && (channels == 1 || channels == 3))
        if (p.h16) k_dwt_inv<1, kOutPlanes, true><<<dim3(tx, ty, channels), DWT_THREADS, inv_smem(1), st>>>(p);
        else k_dwt_inv<1, kOutPlanes, false><<<dim3(tx, ty, channels), DWT_THREADS, inv_smem(1), st>>>(p);
    else if (out_mode == kOutRgb && channels == 3)
        if (p.h16) k_dwt_inv<3, kOutRgb, true><<<dim3(tx, ty, 1), DWT_THREADS, inv_smem(3), st>>>(p);
        else k_dwt_inv<3, kOutRgb, false><<<dim3(tx, ty, 1), DWT_THREADS, inv_smem(3), st>>>(p);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace wema

namespace wema {

// ---- the autotuner's trial of the batched luma kernels' variants: the
// forward level-0 transform of a 3840 x 4320 RGB24 frame (two 2160-row frames'
// worth of tiles) and the inverse level-0 transform of its planes, each
// variant timed over five launches after one warm-up through the batched
// launch path (one task); the fastest of each is kept for the device.
cudaError_t dwt_autotune(int dev, float fwd_ms[9], float inv_ms[9], int* fwd_best, int* inv_best) {
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return e;
    const int W = 3840, H = 4320, SW = W / 2, SH = H / 2;   // level 0 of a 3840x4320 luma frame
    const size_t P = (size_t)W * H, N = (size_t)SW * SH;
    uint8_t* rgb = nullptr;
    float *coef = nullptr, *delta = nullptr, *ll = nullptr, *out = nullptr, *thr = nullptr;
    void *dp = nullptr, *dmap = nullptr, *state = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    const int keep_f = dwt_variant(dev, 0), keep_i = dwt_variant(dev, 1);
    auto done = [&](cudaError_t r) {
        for (void* p : {(void*)rgb, (void*)coef, (void*)delta, (void*)ll, (void*)out, (void*)thr, dp, dmap, state})
            if (p) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
        if (r != cudaSuccess) {                   // leave the device's choices as they were
            dwt_set_variant(dev, 0, keep_f);
            dwt_set_variant(dev, 1, keep_i);
        }
        return r;
    };
    if ((e = cudaMalloc(&rgb, 3 * P)) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&coef, 3 * N * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&delta, 3 * N * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&ll, N * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&out, P * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&thr, 8 * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&state, 3 * N * sizeof(float4))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(state, 0, 3 * N * sizeof(float4))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&dp, sizeof(FwdLevelParams) + sizeof(InvLevelParams))) != cudaSuccess) return done(e);
    if ((e = cudaMalloc(&dmap, 8 * sizeof(int))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(rgb, 0x5a, 3 * P)) != cudaSuccess) return done(e);
    if ((e = cudaMemset(delta, 0, 3 * N * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaMemset(thr, 0, 8 * sizeof(float))) != cudaSuccess) return done(e);
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return done(e);
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) return done(e);
    if ((e = dwt_prepare_device()) != cudaSuccess) return done(e);
    FwdLevelParams fp{};
    fp.iw = W; fp.ih = H; fp.sw = SW; fp.sh = SH; fp.n = (long long)N;
    fp.vec_end = (long long)P;
    fp.src_u8 = rgb;
    fp.coef[0] = coef;
    fp.ll_out[0] = ll;
    // the steady batched forward runs the IIR step on each coefficient it
    // writes: time that kernel (a stable test biquad, poles at 0.9)
    fp.iir_state[0] = state;
    fp.iir_delta[0] = delta;
    const float bq[5] = {0.1f, 0.0f, -0.1f, -1.8f, 0.81f};
    for (int k = 0; k < 10; k++) fp.iir_c[k] = bq[k % 5];
    fp.iir_off6 = 0;
    fp.iir_simd_end = 6 * (long long)N;
    InvLevelParams ip{};
    ip.ow = W; ip.oh = H; ip.sw = SW; ip.sh = SH; ip.n = (long long)N;
    ip.ll[0] = ll;
    ip.coef[0] = coef;
    ip.delta[0] = delta;
    ip.thr = thr;
    ip.alpha[0] = 1.0f;
    ip.out_planes[0] = out;
    if ((e = cudaMemcpy(dp, &fp, sizeof fp, cudaMemcpyHostToDevice)) != cudaSuccess) return done(e);
    char* dpi = static_cast<char*>(dp) + sizeof(FwdLevelParams);
    if ((e = cudaMemcpy(dpi, &ip, sizeof ip, cudaMemcpyHostToDevice)) != cudaSuccess) return done(e);
    unsigned gx, gy;
    const unsigned fblocks = dwt_fwd_grid(fp, 1, gx, gy);
    const int fmap[5] = {1, 0, (int)fblocks, (int)gx, (int)gy};
    const unsigned iblocks = dwt_inv_grid(ip, 1, gx, gy);
    const int imap[5] = {1, 0, (int)iblocks, (int)gx, (int)gy};
    int* map = static_cast<int*>(dmap);
    for (int inv = 0; inv < 2; inv++) {
        if ((e = cudaMemcpy(map, inv ? imap : fmap, sizeof fmap, cudaMemcpyHostToDevice)) != cudaSuccess)
            return done(e);
        float* ms = inv ? inv_ms : fwd_ms;
        int best = 0;
        for (int v = 0; v < kDwtVariants; v++) {
            dwt_set_variant(dev, inv, v);
            for (int rep = 0; rep < 6; rep++) {
                if (rep == 1 && (e = cudaEventRecord(e0, st)) != cudaSuccess) return done(e);
                e = inv ? launch_dwt_inv_multi(1, kOutPlanes, (const InvLevelParams*)dpi, map, iblocks, false, st)
                        : launch_dwt_fwd_multi(kSrcRgbU8, 1, (const FwdLevelParams*)dp, map, fblocks, false, st);
                if (e != cudaSuccess) return done(e);
            }
            if ((e = cudaEventRecord(e1, st)) != cudaSuccess) return done(e);
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return done(e);
            float t = 0.f;
            if ((e = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) return done(e);
            ms[v] = t / 5.f;
            if (ms[v] < ms[best]) best = v;
        }
        dwt_set_variant(dev, inv, best);
        (inv ? *inv_best : *fwd_best) = best;
    }
    return done(cudaSuccess);
}

}  // namespace wema
