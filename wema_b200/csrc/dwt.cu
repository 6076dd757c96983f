// dwt.cu - 2D CDF 9/7 lifting DWT, forward and inverse, one fused kernel per
// pyramid level.
//
// A CTA owns a tile of TP x TP subband pairs (TP = 27) of one channel and
// stages a 64 x 64 sample region - the tile's 54 samples plus a 4-sample
// halo before and a 6-sample halo after, clipped at the image - in shared
// memory.  Lifting runs in registers: a warp takes one line of the region,
// lane k holding the sample pair (2k, 2k+1), and each of the four lifting
// steps is one warp shuffle for the neighbour plus one FMA.  Rows first, then
// the tile's columns (forward); columns over the whole region, then the
// tile's rows (inverse).  Three block barriers per tile.
//
// Every output depends only on samples within 4 of it, so with the halo each
// tile is independent: at the image border the reference's whole-sample
// mirror applies (dwt.c:63-98, 126-160); at a tile border the halo is real
// data, and the garbage that the staged segment's own ends produce moves
// inward by at most two lanes, all inside the halo.  Arithmetic is the
// reference's: x = fma(left + right, c, x), scalings as separate multiplies
// (dwt.c:45-170 as GCC -Ofast evaluates it), so coefficients are bit-exact.
#include "common.cuh"
#include "kernels.h"

namespace wema {

constexpr int TP = 27;                 // subband pairs per tile side
constexpr int SEG = 64;                // staged samples per line (32 lanes x 2)
constexpr int HALO_L = 4;
constexpr int RS = SEG + 1;            // shared-memory row stride (odd: column reads spread banks)
constexpr int DWT_THREADS = 256;
constexpr int NWARP = DWT_THREADS / 32;
constexpr unsigned FULL = 0xffffffffu;

// first staged sample of the tile starting at pair p0 (even)
__device__ __forceinline__ int seg_start(int p0) { return p0 == 0 ? 0 : 2 * p0 - HALO_L; }

// Forward lifting of one line: lane holds samples s = g0 + 2*lane (even) and
// s + 1 of a line of n samples.
__device__ __forceinline__ void lift_fwd(float& e, float& o, int s, int n) {
    const bool r_ok = s + 2 < n;     // predict: right even neighbour s+2
    const bool l_ok = s >= 1;        // update: left odd neighbour s-1
    const bool ro_ok = s + 1 < n;    // update: right odd neighbour s+1
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
__device__ __forceinline__ void lift_inv(float& e, float& o, int s, int n) {
    const bool r_ok = s + 2 < n;
    const bool l_ok = s >= 1;
    const bool ro_ok = s + 1 < n;
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

__device__ __forceinline__ float src_value(const FwdLevelParams& p, const float* lut, int mode,
                                           int c, int chans, long long pi) {
    if (mode == kSrcPlanes) return p.src_planes[c][pi];
    float r, g, b;
    if (mode == kSrcRgbU8) {
        const uint8_t* q = p.src_u8 + 3 * pi;
        r = lut[q[0]]; g = lut[q[1]]; b = lut[q[2]];
    } else {
        const float* q = p.src_f32 + 3 * pi;
        r = q[0]; g = q[1]; b = q[2];
    }
    const bool vec = pi < p.vec_end;
    if (chans == 1) return vec ? luma_vec(r, g, b) : luma_tail(r, g, b);
    float y, cb, cr;
    if (vec) ycbcr_vec(r, g, b, y, cb, cr);
    else ycbcr_tail(r, g, b, y, cb, cr);
    return c == 0 ? y : (c == 1 ? cb : cr);
}

// ----------------------------------------------------------------- forward
// grid: (tiles_x, tiles_y, channels); one channel per CTA
template <int MODE>
__global__ void __launch_bounds__(DWT_THREADS) k_dwt_fwd(FwdLevelParams p, int chans) {
    __shared__ float sm[SEG * RS];
    __shared__ float lut[256];
    const int c = blockIdx.z;
    if (MODE == kSrcRgbU8)
        for (int i = threadIdx.x; i < 256; i += DWT_THREADS) lut[i] = __fdiv_rn((float)i, 255.0f);
    const int iw = p.iw, ih = p.ih, sw = p.sw, sh = p.sh;
    const int px0 = blockIdx.x * TP, py0 = blockIdx.y * TP;
    const int rx0 = seg_start(px0), ry0 = seg_start(py0);
    const int RW = min(SEG, iw - rx0), RH = min(SEG, ih - ry0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (MODE == kSrcRgbU8) __syncthreads();

    // staging: all PER loads of a thread are issued before any is used
    constexpr int PER = SEG * SEG / DWT_THREADS;
    float v[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int k = threadIdx.x + q * DWT_THREADS;
        const int ly = k >> 6, lx = k & 63;
        v[q] = (ly < RH && lx < RW)
                   ? src_value(p, lut, MODE, c, chans, (long long)(ry0 + ly) * iw + (rx0 + lx))
                   : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int k = threadIdx.x + q * DWT_THREADS;
        const int ly = k >> 6, lx = k & 63;
        if (ly < RH && lx < RW) {
            sm[ly * RS + lx] = v[q];
            if (MODE != kSrcPlanes && p.plane_out[c])
                p.plane_out[c][(long long)(ry0 + ly) * iw + (rx0 + lx)] = v[q];
        }
    }
    __syncthreads();

    if (iw >= 2) {   // rows: every staged row
        for (int ly = warp; ly < RH; ly += NWARP) {
            float* row = sm + ly * RS;
            float e = row[2 * lane], o = row[2 * lane + 1];
            lift_fwd(e, o, rx0 + 2 * lane, iw);
            if (2 * lane < RW) row[2 * lane] = e;
            if (2 * lane + 1 < RW) row[2 * lane + 1] = o;
        }
        __syncthreads();
    }
    const int cx0 = 2 * px0 - rx0, cx1 = min(2 * (px0 + TP), iw) - rx0;
    if (ih >= 2) {   // columns: the tile's own
        for (int lx = cx0 + warp; lx < cx1; lx += NWARP) {
            float* col = sm + lx;
            float e = col[(2 * lane) * RS], o = col[(2 * lane + 1) * RS];
            lift_fwd(e, o, ry0 + 2 * lane, ih);
            if (2 * lane < RH) col[(2 * lane) * RS] = e;
            if (2 * lane + 1 < RH) col[(2 * lane + 1) * RS] = o;
        }
        __syncthreads();
    }

    // quadrants: LL (even,even), HL (odd x), LH (odd y), HH; stale entries of
    // odd-sized levels take the previous level's value at the same index
    const int ni = min(TP, sw - px0), nj = min(TP, sh - py0);
    float* bands = p.coef[c];
    const float* prev = p.prev[c];
    for (int k = threadIdx.x; k < ni * nj; k += DWT_THREADS) {
        const int jj = k / ni, ii = k - jj * ni;
        const int i = px0 + ii, j = py0 + jj;
        const int lx = 2 * i - rx0, ly = 2 * j - ry0;
        const long long o = (long long)j * sw + i;
        const bool hx = 2 * i + 1 < iw, hy = 2 * j + 1 < ih;
        p.ll_out[c][o] = sm[ly * RS + lx];
        bands[o] = hy ? sm[(ly + 1) * RS + lx] : (prev ? prev[o] : 0.0f);                    // LH
        bands[p.n + o] = (hx && hy) ? sm[(ly + 1) * RS + lx + 1]
                                    : (prev ? prev[p.prev_n + o] : 0.0f);                 // HH
        bands[2 * p.n + o] = hx ? sm[ly * RS + lx + 1] : (prev ? prev[2 * p.prev_n + o] : 0.0f); // HL
    }
}

// ----------------------------------------------------------------- inverse
// C == 1: grid (tiles_x, tiles_y, channels), planes out.
// C == 3: one CTA per tile does all three channels (YCbCr -> RGB at level 0).
template <int C, int OUT>
__global__ void __launch_bounds__(DWT_THREADS) k_dwt_inv(InvLevelParams p) {
    extern __shared__ float dyn[];
    float(*smem)[SEG * RS] = reinterpret_cast<float(*)[SEG * RS]>(dyn);
    const int ow = p.ow, oh = p.oh, sw = p.sw;
    const int px0 = blockIdx.x * TP, py0 = blockIdx.y * TP;
    const int rx0 = seg_start(px0), ry0 = seg_start(py0);
    const int RW = min(SEG, ow - rx0), RH = min(SEG, oh - ry0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = (C == 1) ? blockIdx.z : 0;

    // interleave LL / HL / LH / HH into the sample grid; bands are amplified
    // on the way in.  Coefficient and delta loads of all PER samples of a
    // thread are issued before any is used.
    constexpr int PER = SEG * SEG / DWT_THREADS;
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
        const int ch = c0 + cc;
        const float thr = p.thr[ch];
        const float al = p.alpha[ch];
        float a[PER], d[PER];
        bool band[PER];
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int k = threadIdx.x + q * DWT_THREADS;
            const int ly = k >> 6, lx = k & 63;
            a[q] = 0.0f;
            d[q] = 0.0f;
            band[q] = false;
            if (ly < RH && lx < RW) {
                const int gy = ry0 + ly, gx = rx0 + lx;
                const long long o = (long long)(gy >> 1) * sw + (gx >> 1);
                const int qd = (gx & 1) | ((gy & 1) << 1);
                if (qd == 0) {
                    a[q] = p.ll[ch][o];
                } else {
                    // LH (qd 2), HH (qd 3), HL (qd 1)
                    const long long bo = (qd == 1 ? 2 * p.n : (qd == 2 ? 0 : p.n)) + o;
                    a[q] = p.coef[ch][bo];
                    d[q] = p.delta[ch][bo];
                    band[q] = true;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int k = threadIdx.x + q * DWT_THREADS;
            const int ly = k >> 6, lx = k & 63;
            if (ly < RH && lx < RW) {
                float x = a[q];
                if (band[q] && fabsf(x) > thr) x = __fmaf_rn(d[q], al, x);
                smem[cc][ly * RS + lx] = x;
            }
        }
    }
    __syncthreads();
    if (oh >= 2) {   // columns over the whole staged region
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int lx = warp; lx < RW; lx += NWARP) {
                float* col = smem[cc] + lx;
                float e = col[(2 * lane) * RS], o = col[(2 * lane + 1) * RS];
                lift_inv(e, o, ry0 + 2 * lane, oh);
                if (2 * lane < RH) col[(2 * lane) * RS] = e;
                if (2 * lane + 1 < RH) col[(2 * lane + 1) * RS] = o;
            }
        __syncthreads();
    }
    const int ty0 = 2 * py0 - ry0, ty1 = min(2 * (py0 + TP), oh) - ry0;
    const int tx0 = 2 * px0 - rx0, tx1 = min(2 * (px0 + TP), ow) - rx0;
    if (ow >= 2) {   // rows of the tile
#pragma unroll
        for (int cc = 0; cc < C; cc++)
            for (int ly = ty0 + warp; ly < ty1; ly += NWARP) {
                float* row = smem[cc] + ly * RS;
                float e = row[2 * lane], o = row[2 * lane + 1];
                lift_inv(e, o, rx0 + 2 * lane, ow);
                if (2 * lane < RW) row[2 * lane] = e;
                if (2 * lane + 1 < RW) row[2 * lane + 1] = o;
            }
        __syncthreads();
    }
    const int nx = tx1 - tx0, ny = ty1 - ty0;
    for (int k = threadIdx.x; k < nx * ny; k += DWT_THREADS) {
        const int yy = k / nx, xx = k - yy * nx;
        const int ly = ty0 + yy, lx = tx0 + xx;
        const long long pi = (long long)(ry0 + ly) * ow + (rx0 + lx);
        if (OUT == kOutPlanes) {
#pragma unroll
            for (int cc = 0; cc < C; cc++) p.out_planes[c0 + cc][pi] = smem[cc][ly * RS + lx];
        } else {
            const float y = smem[0][ly * RS + lx];
            const float cb = smem[C > 1 ? 1 : 0][ly * RS + lx];
            const float cr = smem[C > 2 ? 2 : 0][ly * RS + lx];
            if (p.out_planes[0]) {
                p.out_planes[0][pi] = y;
                p.out_planes[1][pi] = cb;
                p.out_planes[2][pi] = cr;
            }
            float r, g, b;
            ycbcr_to_rgb(y, cb, cr, r, g, b);
            if (p.out_u8) {
                uint8_t* d = p.out_u8 + 3 * pi;
                d[0] = quant_u8(r); d[1] = quant_u8(g); d[2] = quant_u8(b);
            }
            if (p.out_f32) {
                float* d = p.out_f32 + 3 * pi;
                d[0] = r; d[1] = g; d[2] = b;
            }
        }
    }
}

// ----------------------------------------------------------------- launch

size_t dwt_smem_bytes(int C) { return (size_t)C * SEG * RS * sizeof(float); }

static unsigned tiles_of(int pairs) { return (unsigned)((pairs + TP - 1) / TP); }

// the three-channel inverse needs more than the 48 KB default; call once per device
cudaError_t dwt_prepare_device() {
    return cudaFuncSetAttribute(k_dwt_inv<3, kOutRgb>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dwt_smem_bytes(3));
}

cudaError_t launch_dwt_fwd(int mode, int channels, const FwdLevelParams& p, cudaStream_t st) {
    if (channels != 1 && channels != 3) return cudaErrorInvalidValue;
    dim3 grid(tiles_of(p.sw), tiles_of(p.sh), channels);
    switch (mode) {
        case kSrcPlanes: k_dwt_fwd<kSrcPlanes><<<grid, DWT_THREADS, 0, st>>>(p, channels); break;
        case kSrcRgbU8: k_dwt_fwd<kSrcRgbU8><<<grid, DWT_THREADS, 0, st>>>(p, channels); break;
        case kSrcRgbF32: k_dwt_fwd<kSrcRgbF32><<<grid, DWT_THREADS, 0, st>>>(p, channels); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dwt_inv(int channels, int out_mode, const InvLevelParams& p, cudaStream_t st) {
    const unsigned tx = tiles_of((p.ow + 1) / 2), ty = tiles_of((p.oh + 1) / 2);
    if (out_mode == kOutPlanes && (channels == 1 || channels == 3))
        k_dwt_inv<1, kOutPlanes><<<dim3(tx, ty, channels), DWT_THREADS, dwt_smem_bytes(1), st>>>(p);
    else if (out_mode == kOutRgb && channels == 3)
        k_dwt_inv<3, kOutRgb><<<dim3(tx, ty, 1), DWT_THREADS, dwt_smem_bytes(3), st>>>(p);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace wema
