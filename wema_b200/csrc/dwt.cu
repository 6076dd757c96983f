// dwt.cu - 2D CDF 9/7 lifting DWT, forward and inverse, one fused kernel per
// pyramid level.
//
// A CTA owns a tile of TP x TP subband pairs.  It stages the tile plus a
// halo of input samples in shared memory (interleaved layout: even sample =
// low-pass, odd sample = high-pass), runs the four lifting steps along rows,
// scales, runs them along columns, and writes the four quadrants.  Every
// output sample depends only on samples within +-4 (forward) / +-4
// (inverse), so the halo makes each tile independent: at the image border
// the reference's whole-sample mirror applies (dwt.c:63-98 / 126-160), at a
// tile border the halo samples are used and whatever the halo's own outer
// edge computes never reaches the tile.  Per-sample arithmetic is the
// reference's: x = fma(left + right, c, x) with the scalings as separate
// multiplies (dwt.c:45-170 as GCC -Ofast evaluates it).
#include "common.cuh"
#include "kernels.h"

namespace wema {

constexpr int TP = 32;               // subband pairs per tile side
constexpr int FWD_HALO_L = 4, FWD_HALO_R = 6;
constexpr int INV_HALO = 4;
constexpr int RMAX = 2 * TP + 10;    // region side (forward; inverse needs 2TP+8)
constexpr int RSTRIDE = RMAX + 1;    // padded row stride in shared memory
constexpr int DWT_THREADS = 256;

// neighbour of global sample s at distance +-1: whole-sample mirror at the
// image ends, then clamped into the staged region [r0, r1).
__device__ __forceinline__ int nb(int s, int d, int n, int r0, int r1) {
    int t = s + d;
    if (t < 0 || t >= n) t = s - d;
    return min(max(t, r0), r1 - 1);
}

// One lifting step along rows: samples of parity `par` in [r0, r1), lines
// [l0, l1) of the tile (each line is a shared-memory row).
__device__ __forceinline__ void step_rows(float* sm, int l0, int l1, int r0, int r1, int n,
                                          int par, float c) {
    const int first = r0 + ((r0 & 1) != par);
    const int cnt = first < r1 ? (r1 - first + 1) / 2 : 0;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int l = l0 + ty; l < l1; l += DWT_THREADS / 32) {
        float* row = sm + l * RSTRIDE - r0;
        for (int k = tx; k < cnt; k += 32) {
            int s = first + 2 * k;
            float a = row[nb(s, -1, n, r0, r1)], b = row[nb(s, 1, n, r0, r1)];
            row[s] = __fmaf_rn(__fadd_rn(a, b), c, row[s]);
        }
    }
    __syncthreads();
}

// One lifting step along columns: samples of parity `par` in [r0, r1) of the
// columns [c0, c1) (local column indices).
__device__ __forceinline__ void step_cols(float* sm, int c0, int c1, int r0, int r1, int n,
                                          int par, float c) {
    const int first = r0 + ((r0 & 1) != par);
    const int cnt = first < r1 ? (r1 - first + 1) / 2 : 0;
    const int ncol = c1 - c0;
    for (int k = threadIdx.x; k < cnt * ncol; k += DWT_THREADS) {
        int s = first + 2 * (k / ncol);
        int col = c0 + k % ncol;
        float* cp = sm + col - r0 * RSTRIDE;
        float a = cp[nb(s, -1, n, r0, r1) * RSTRIDE], b = cp[nb(s, 1, n, r0, r1) * RSTRIDE];
        cp[s * RSTRIDE] = __fmaf_rn(__fadd_rn(a, b), c, cp[s * RSTRIDE]);
    }
    __syncthreads();
}

// ----------------------------------------------------------------- forward

template <int MODE, int C>
__global__ void __launch_bounds__(DWT_THREADS) k_dwt_fwd(FwdLevelParams p) {
    extern __shared__ float smem[];
    __shared__ float lut[256];
    if (MODE == kSrcRgbU8)
        for (int i = threadIdx.x; i < 256; i += DWT_THREADS) lut[i] = __fdiv_rn((float)i, 255.0f);

    const int iw = p.iw, ih = p.ih, sw = p.sw, sh = p.sh;
    const int px0 = blockIdx.x * TP, py0 = blockIdx.y * TP;
    const int rx0 = max(2 * px0 - FWD_HALO_L, 0), rx1 = min(2 * (px0 + TP) + FWD_HALO_R, iw);
    const int ry0 = max(2 * py0 - FWD_HALO_L, 0), ry1 = min(2 * (py0 + TP) + FWD_HALO_R, ih);
    const int RW = rx1 - rx0, RH = ry1 - ry0;
    const int chan_sz = RMAX * RSTRIDE;
    __syncthreads();

    // stage the region (level 0 converts RGB to Y or Y/Cb/Cr on the fly)
    for (int k = threadIdx.x; k < RW * RH; k += DWT_THREADS) {
        const int ly = k / RW, lx = k - ly * RW;
        const int gy = ry0 + ly, gx = rx0 + lx;
        const long long pi = (long long)gy * iw + gx;
        float v[3];
        if (MODE == kSrcPlanes) {
#pragma unroll
            for (int c = 0; c < C; c++) v[c] = p.src_planes[c][pi];
        } else {
            float r, g, b;
            if (MODE == kSrcRgbU8) {
                const uint8_t* q = p.src_u8 + 3 * pi;
                r = lut[q[0]]; g = lut[q[1]]; b = lut[q[2]];
            } else {
                const float* q = p.src_f32 + 3 * pi;
                r = q[0]; g = q[1]; b = q[2];
            }
            const bool vec = pi < p.vec_end;
            if (C == 1) {
                v[0] = vec ? luma_vec(r, g, b) : luma_tail(r, g, b);
            } else {
                if (vec) ycbcr_vec(r, g, b, v[0], v[1], v[2]);
                else ycbcr_tail(r, g, b, v[0], v[1], v[2]);
            }
            if (p.plane_out[0]) {   // keep the input planes (host inspection)
#pragma unroll
                for (int c = 0; c < C; c++) p.plane_out[c][pi] = v[c];
            }
        }
#pragma unroll
        for (int c = 0; c < C; c++) smem[c * chan_sz + ly * RSTRIDE + lx] = v[c];
    }
    __syncthreads();

    // rows: all staged rows, global sample range [rx0, rx1) of length iw
    if (iw >= 2) {
#pragma unroll
        for (int c = 0; c < C; c++) {
            float* sm = smem + c * chan_sz;
            step_rows(sm, 0, RH, rx0, rx1, iw, 1, kAlpha);
            step_rows(sm, 0, RH, rx0, rx1, iw, 0, kBeta);
            step_rows(sm, 0, RH, rx0, rx1, iw, 1, kGamma);
            step_rows(sm, 0, RH, rx0, rx1, iw, 0, kDelta);
        }
        for (int k = threadIdx.x; k < RW * RH; k += DWT_THREADS) {
            const int ly = k / RW, lx = k - ly * RW;
            const float s = ((rx0 + lx) & 1) ? kK : kKInv;
#pragma unroll
            for (int c = 0; c < C; c++) {
                float* q = smem + c * chan_sz + ly * RSTRIDE + lx;
                *q = __fmul_rn(*q, s);
            }
        }
        __syncthreads();
    }
    // columns: only the tile's own columns are needed from here on
    const int cx0 = 2 * px0 - rx0, cx1 = min(2 * (px0 + TP), iw) - rx0;
    if (ih >= 2 && cx1 > cx0) {
#pragma unroll
        for (int c = 0; c < C; c++) {
            float* sm = smem + c * chan_sz;
            step_cols(sm, cx0, cx1, ry0, ry1, ih, 1, kAlpha);
            step_cols(sm, cx0, cx1, ry0, ry1, ih, 0, kBeta);
            step_cols(sm, cx0, cx1, ry0, ry1, ih, 1, kGamma);
            step_cols(sm, cx0, cx1, ry0, ry1, ih, 0, kDelta);
        }
    }

    // quadrants; column scaling folded into the store
    const int ni = min(TP, sw - px0), nj = min(TP, sh - py0);
    const bool cs = ih >= 2;
    for (int k = threadIdx.x; k < ni * nj; k += DWT_THREADS) {
        const int jj = k / ni, ii = k - jj * ni;
        const int i = px0 + ii, j = py0 + jj;
        const int lx = 2 * i - rx0, ly = 2 * j - ry0;
        const long long o = (long long)j * sw + i;
        const bool hx = 2 * i + 1 < iw, hy = 2 * j + 1 < ih;
#pragma unroll
        for (int c = 0; c < C; c++) {
            const float* sm = smem + c * chan_sz;
            float ll = sm[ly * RSTRIDE + lx];
            p.ll_out[c][o] = cs ? __fmul_rn(ll, kKInv) : ll;
            float* bands = p.coef[c];          // LH, HH, HL of this level
            const float* prev = p.prev[c];     // previous level's bands (stale source)
            float lh, hh, hl;
            if (hy) lh = __fmul_rn(sm[(ly + 1) * RSTRIDE + lx], kK);
            else lh = prev ? prev[o] : 0.0f;
            if (hx && hy) hh = __fmul_rn(sm[(ly + 1) * RSTRIDE + lx + 1], kK);
            else hh = prev ? prev[p.prev_n + o] : 0.0f;
            if (hx) { float v = sm[ly * RSTRIDE + lx + 1]; hl = cs ? __fmul_rn(v, kKInv) : v; }
            else hl = prev ? prev[2 * p.prev_n + o] : 0.0f;
            bands[o] = lh;
            bands[p.n + o] = hh;
            bands[2 * p.n + o] = hl;
        }
    }
}

// ----------------------------------------------------------------- inverse

template <int C, int OUT>
__global__ void __launch_bounds__(DWT_THREADS) k_dwt_inv(InvLevelParams p) {
    extern __shared__ float smem[];
    const int ow = p.ow, oh = p.oh, sw = p.sw;
    const int px0 = blockIdx.x * TP, py0 = blockIdx.y * TP;
    const int rx0 = max(2 * px0 - INV_HALO, 0), rx1 = min(2 * (px0 + TP) + INV_HALO, ow);
    const int ry0 = max(2 * py0 - INV_HALO, 0), ry1 = min(2 * (py0 + TP) + INV_HALO, oh);
    const int RW = rx1 - rx0, RH = ry1 - ry0;
    const int chan_sz = RMAX * RSTRIDE;
    const bool cs = oh >= 2, rs = ow >= 2;

    // interleave LL / HL / LH / HH into the sample grid, column scale folded in
    for (int k = threadIdx.x; k < RW * RH; k += DWT_THREADS) {
        const int ly = k / RW, lx = k - ly * RW;
        const int gy = ry0 + ly, gx = rx0 + lx;
        const long long o = (long long)(gy >> 1) * sw + (gx >> 1);
        const int q = (gx & 1) | ((gy & 1) << 1);
#pragma unroll
        for (int c = 0; c < C; c++) {
            float v;
            if (q == 0) v = p.ll[c][o];
            else if (q == 1) v = p.coef[c][2 * p.n + o];   // HL
            else if (q == 2) v = p.coef[c][o];             // LH
            else v = p.coef[c][p.n + o];                   // HH
            if (cs) v = __fmul_rn(v, (gy & 1) ? kKInv : kK);
            smem[c * chan_sz + ly * RSTRIDE + lx] = v;
        }
    }
    __syncthreads();
    if (cs) {
#pragma unroll
        for (int c = 0; c < C; c++) {
            float* sm = smem + c * chan_sz;
            step_cols(sm, 0, RW, ry0, ry1, oh, 0, -kDelta);
            step_cols(sm, 0, RW, ry0, ry1, oh, 1, -kGamma);
            step_cols(sm, 0, RW, ry0, ry1, oh, 0, -kBeta);
            step_cols(sm, 0, RW, ry0, ry1, oh, 1, -kAlpha);
        }
    }
    const int ty0 = 2 * py0 - ry0, ty1 = min(2 * (py0 + TP), oh) - ry0;
    if (rs) {
        for (int k = threadIdx.x; k < RW * (ty1 - ty0); k += DWT_THREADS) {
            const int ly = ty0 + k / RW, lx = k % RW;
            const float s = ((rx0 + lx) & 1) ? kKInv : kK;
#pragma unroll
            for (int c = 0; c < C; c++) {
                float* q = smem + c * chan_sz + ly * RSTRIDE + lx;
                *q = __fmul_rn(*q, s);
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < C; c++) {
            float* sm = smem + c * chan_sz;
            step_rows(sm, ty0, ty1, rx0, rx1, ow, 0, -kDelta);
            step_rows(sm, ty0, ty1, rx0, rx1, ow, 1, -kGamma);
            step_rows(sm, ty0, ty1, rx0, rx1, ow, 0, -kBeta);
            step_rows(sm, ty0, ty1, rx0, rx1, ow, 1, -kAlpha);
        }
    }
    const int tx0 = 2 * px0 - rx0, tx1 = min(2 * (px0 + TP), ow) - rx0;
    const int nx = tx1 - tx0, ny = ty1 - ty0;
    for (int k = threadIdx.x; k < nx * ny; k += DWT_THREADS) {
        const int ly = ty0 + k / nx, lx = tx0 + k % nx;
        const long long pi = (long long)(ry0 + ly) * ow + (rx0 + lx);
        if (OUT == kOutPlanes) {
#pragma unroll
            for (int c = 0; c < C; c++) p.out_planes[c][pi] = smem[c * chan_sz + ly * RSTRIDE + lx];
        } else {
            // colour mode, level 0: YCbCr -> RGB with clamp (wema.c:80-102)
            float y = smem[ly * RSTRIDE + lx];
            float cb = smem[chan_sz + ly * RSTRIDE + lx];
            float cr = smem[2 * chan_sz + ly * RSTRIDE + lx];
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

size_t dwt_smem_bytes(int C) { return (size_t)C * RMAX * RSTRIDE * sizeof(float); }

static dim3 tiles(int w, int h) { return dim3((w + TP - 1) / TP, (h + TP - 1) / TP); }

template <int MODE, int C>
static cudaError_t fwd_launch(const FwdLevelParams& p, cudaStream_t st) {
    k_dwt_fwd<MODE, C><<<tiles(p.sw, p.sh), DWT_THREADS, dwt_smem_bytes(C), st>>>(p);
    return cudaGetLastError();
}

template <int C, int OUT>
static cudaError_t inv_launch(const InvLevelParams& p, cudaStream_t st) {
    const int pw = (p.ow + 1) / 2, ph = (p.oh + 1) / 2;
    k_dwt_inv<C, OUT><<<tiles(pw, ph), DWT_THREADS, dwt_smem_bytes(C), st>>>(p);
    return cudaGetLastError();
}

// Opts every instantiation into the shared memory it needs (more than the
// 48 KB default for three channels); call once per device.
cudaError_t dwt_prepare_device() {
    const int a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaSuccess;
#define WEMA_ATTR(fn, c) if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, (cudaFuncAttribute)a, (int)dwt_smem_bytes(c))
    WEMA_ATTR((k_dwt_fwd<kSrcPlanes, 1>), 1);
    WEMA_ATTR((k_dwt_fwd<kSrcRgbU8, 1>), 1);
    WEMA_ATTR((k_dwt_fwd<kSrcRgbF32, 1>), 1);
    WEMA_ATTR((k_dwt_fwd<kSrcPlanes, 3>), 3);
    WEMA_ATTR((k_dwt_fwd<kSrcRgbU8, 3>), 3);
    WEMA_ATTR((k_dwt_fwd<kSrcRgbF32, 3>), 3);
    WEMA_ATTR((k_dwt_inv<1, kOutPlanes>), 1);
    WEMA_ATTR((k_dwt_inv<3, kOutPlanes>), 3);
    WEMA_ATTR((k_dwt_inv<3, kOutRgb>), 3);
#undef WEMA_ATTR
    return e;
}

cudaError_t launch_dwt_fwd(int mode, int channels, const FwdLevelParams& p, cudaStream_t st) {
    if (channels == 1) {
        switch (mode) {
            case kSrcPlanes: return fwd_launch<kSrcPlanes, 1>(p, st);
            case kSrcRgbU8: return fwd_launch<kSrcRgbU8, 1>(p, st);
            case kSrcRgbF32: return fwd_launch<kSrcRgbF32, 1>(p, st);
        }
    } else if (channels == 3) {
        switch (mode) {
            case kSrcPlanes: return fwd_launch<kSrcPlanes, 3>(p, st);
            case kSrcRgbU8: return fwd_launch<kSrcRgbU8, 3>(p, st);
            case kSrcRgbF32: return fwd_launch<kSrcRgbF32, 3>(p, st);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_dwt_inv(int channels, int out_mode, const InvLevelParams& p, cudaStream_t st) {
    if (channels == 1 && out_mode == kOutPlanes) return inv_launch<1, kOutPlanes>(p, st);
    if (channels == 3 && out_mode == kOutPlanes) return inv_launch<3, kOutPlanes>(p, st);
    if (channels == 3 && out_mode == kOutRgb) return inv_launch<3, kOutRgb>(p, st);
    return cudaErrorInvalidValue;
}

}  // namespace wema
