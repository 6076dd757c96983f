// kernels.h - launch interface of the sm_100a kernels (host side of csrc/).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace wema {

// ---- DWT (dwt.cu) --------------------------------------------------------
enum { kSrcPlanes = 0, kSrcRgbU8 = 1, kSrcRgbF32 = 2 };
enum { kOutPlanes = 0, kOutRgb = 1 };

struct FwdLevelParams {
    int iw, ih;                 // level input size
    int sw, sh;                 // subband size
    long long n;                // sw*sh
    long long vec_end;          // level 0: pixels below use the vector-body luma form
    const float* src_planes[3]; // levels >= 1: input planes (previous LL)
    const uint8_t* src_u8;      // level 0: interleaved RGB24
    const float* src_f32;       // level 0: interleaved float RGB
    float* plane_out[3];        // level 0, optional: converted Y / Cb / Cr planes
    float* coef[3];             // this level's bands LH, HH, HL (n each)
    const float* prev[3];       // previous level's bands (stale entries), or null
    long long prev_n;
    float* ll_out[3];           // LL (next level's input or the lowpass)
    int h16;                    // coef and prev are FP16 planes (src_planes, ll_out stay FP32)
    // the temporal filter's step on each coefficient as it is written (IIR
    // streams after their first frame); iir_state[c] null: off
    void* iir_state[3];         // this level's biquad state (float4, or 2 x double2 with iir_fp64)
    float* iir_delta[3];        // this level's band-passed delta planes
    float iir_c[10];            // {b0,b1,b2,a1,a2} high-pass, then low-pass
    long long iir_off6;         // this level's first 6-slot index
    long long iir_simd_end;     // 6-slot indices from here take the scalar-tail form
    int iir_fp64;
};

struct InvLevelParams {
    int ow, oh;                 // level canvas size (reconstructed image)
    int sw, sh;
    long long n;
    const float* ll[3];         // coarser reconstruction / lowpass (sw x sh)
    const float* coef[3];       // original bands LH, HH, HL of this level
    const float* delta[3];      // band-passed deltas of the same bands
    const float* thr;           // per-channel thresholds (device)
    float alpha[3];             // per-channel level alpha (level 0 already halved)
    float* out_planes[3];       // reconstructed planes (kOutPlanes), optional for kOutRgb
    uint8_t* out_u8;            // kOutRgb: RGB24 output (optional)
    float* out_f32;             // kOutRgb: float RGB output (optional)
    int h16;                    // coef and delta are FP16 planes (ll stays FP32)
    int out16;                  // out_planes are FP16 (the level-0 reconstruction of planes_fp16)
};

cudaError_t dwt_prepare_device();
size_t dwt_smem_bytes(int channels);
cudaError_t launch_dwt_fwd(int src_mode, int channels, const FwdLevelParams& p, cudaStream_t st);
cudaError_t launch_dwt_inv(int channels, int out_mode, const InvLevelParams& p, cudaStream_t st);
// tuning variant (0..8) of the batched luma DWT kernels on a device:
// CTAs per SM {1: the compiler's choice, 3, 4}[v / 3] x lines per warp {2, 4, 8}[v % 3]
int dwt_variant(int dev, int inverse);
bool dwt_set_variant(int dev, int inverse, int v);
void dwt_variant_shape(int v, int* minb, int* lpw);
// times every variant of the forward and inverse level-0 luma kernels, keeps the fastest
cudaError_t dwt_autotune(int dev, float fwd_ms[9], float inv_ms[9], int* fwd_best, int* inv_best);

// ---- exact threshold (threshold.cu) ---------------------------------------
// Views the unique detail planes of one channel as the reference's 6-slot
// flat array and reproduces its vectorised FP32 sum of |x| bit for bit.
struct PyrView {
    const float* coef;          // unique planes (uoff layout); levels == 0: flat array of off6[0]
    int levels;
    long long n[4], uoff[4], off6[5];   // off6[levels] = N6
};

struct ThrScratch {             // device scratch, sized by thr_scratch_bytes; lane-major [8][n_sub]
    double* part;               // sub-chunk sums of |x| (binade prediction)
    double* prefix;             // exclusive FP64 prefixes (first call only)
    int4* candp;                // {primary binade, d0, d1, secondary binade or 0}
    int2* candq;                // secondary {d0, d1}
    int* hist;                  // binade of the running sum at each sub-chunk start, recorded
                                // by the last walk (the next frame's candidates)
    float* lanes;               // [8] final lane sums
    unsigned* counter;          // lanes finished (the last one runs the epilogue)
};
cudaError_t thr_prepare_device();
size_t thr_scratch_bytes(long long n6);
void thr_scratch_bind(ThrScratch& s, void* base, long long n6);
// Writes thr[chan] = threshold of each of `nch` channels (single-frame form
// (sum/N)*0.2, or batch form (0.2/N)*sum); optionally the raw sums.
// use_hist: predict binades from scratch.hist (written by the previous call on
// the same geometry) instead of the FP64 partial sums - skips two kernels.
// h16: the planes are FP16 (planes_fp16 variant): an FP64 sum instead of the
// bit-exact one (the other arguments as above; use_hist unused).
cudaError_t launch_threshold(const PyrView* views, int nch, ThrScratch* scratch, float* thr,
                             float* sums, int batch_form, int use_hist, int h16, cudaStream_t st);

// ---- IIR + amplification (iir.cu) ------------------------------------------
struct IirParams {
    float c[10];                // {b0,b1,b2,a1,a2} high-pass, then low-pass
    int levels;
    long long uoff[5];          // unique-plane level offsets
    long long n[4];
    long long off6[5];
    long long simd_end;         // 6-slot positions >= simd_end take the scalar-tail form
    int h16;                    // coefficient and delta planes are FP16
};
// preseed: run `warmup` iterations with the current coefficients as input
// state: float4 per position, or (fp64) two double2 per position
cudaError_t launch_iir_preseed(const IirParams& p, const float* coef, void* state, int fp64, int warmup,
                               cudaStream_t st);
// one frame: delta = cascade(coef); the amplification is applied where the
// inverse DWT stages the coefficients (launch_dwt_inv) or by launch_amplify
cudaError_t launch_iir(const IirParams& p, const float* coef, void* state, int fp64, float* delta,
                       cudaStream_t st);
// amplified = |coef| > thr ? fma(delta, alpha_l, coef) : coef over all unique
// positions (inspection, and the batch route)
cudaError_t launch_amplify(const IirParams& p, const float* coef, const float* delta,
                           const float* thr, float alpha, float* amplified, cudaStream_t st);

// ---- spatial filter + luma transfer (spatial.cu) ----------------------------
struct TransferParams {
    int w, h;
    long long vec_end;          // guide luma form switch (vector body / tail)
    const uint8_t* src_u8;      // input RGB24 (or null)
    const float* src_f32;       // input float RGB (or null)
    const float* gray_out;      // reconstructed luma
    uint8_t* out_u8;            // output RGB24 (optional)
    float* out_f32;             // output float RGB (optional)
    int edge_aware;             // 1: guided filter r=4 eps=0.01; 0: 5-tap Gaussian
    int seg_rows;               // guided filter: output rows per sweep segment (0: the device's)
    int h16;                    // gray_out is an FP16 plane (planes_fp16)
};
cudaError_t launch_transfer(const TransferParams& p, cudaStream_t st);
cudaError_t spatial_prepare_device();

// copy-through (window mode before the ring is full): out = in
cudaError_t launch_passthrough(const TransferParams& p, cudaStream_t st);

// ---- window (--haar) temporal filter (window.cu) ----------------------------
struct WindowParams {
    long long pu;               // unique positions
    int ws, head;               // window size, ring slot of the oldest sample
    int bilateral;
    int fp16;                   // ring elements are __half (else float)
    int h16;                    // the delta plane written is FP16 (planes_fp16)
    float time_w[256];
};
// coef: FP16 plane when h16 (planes_fp16); ring: __half elements when fp16 (ring_fp16)
cudaError_t launch_ring_push(const float* coef, int h16, void* ring, int fp16, long long pu, int slot,
                             cudaStream_t st);
cudaError_t launch_window(const WindowParams& wp, const void* ring, float* delta,
                          cudaStream_t st);

// ---- batched launches: one launch of a kernel over many streams --------------
// Every launch takes a device array of per-task parameters and a task map
// (multi.cuh); `blocks` is the sum of the tasks' grids.
unsigned dwt_fwd_grid(const FwdLevelParams& p, int channels_z, unsigned& gx, unsigned& gy);
unsigned dwt_inv_grid(const InvLevelParams& p, int channels_z, unsigned& gx, unsigned& gy);
// any16: some task has FP16 planes (planes_fp16); false selects the kernel
// compiled for FP32 planes only
cudaError_t launch_dwt_fwd_multi(int mode, int channels, const FwdLevelParams* d_params,
                                 const int* d_map, unsigned blocks, bool any16, cudaStream_t st);
cudaError_t launch_dwt_inv_multi(int channels, int out_mode, const InvLevelParams* d_params,
                                 const int* d_map, unsigned blocks, bool any16, cudaStream_t st);
size_t thr_args_bytes();
// grids[stage] = {x, y} for stage 0 partials, 1 prefix, 2 monoids, 3 walk
cudaError_t thr_args_fill(void* dst, const PyrView* views, int nch, const ThrScratch* scratch,
                          float* thr, float* sums, int batch_form, int use_hist, unsigned grids[5][2]);
cudaError_t launch_threshold_multi(int stage, const void* d_args, const int* d_map, unsigned blocks,
                                   cudaStream_t st);
// sub-chunks of the 6-slot array that lie wholly in level 0 (0: one level):
// their monoids (stage 2) can run as soon as level 0's forward transform is done
int thr_level0_subchunks(const PyrView& v);
// sets the monoid launch of an args blob to sub-chunks sub0 .. sub1-1 (sub1 < 0:
// to the end); its block count per channel
unsigned thr_args_monoid_part(void* args, int sub0, int sub1);
size_t iir_args_bytes();
unsigned iir_args_fill(void* dst, const IirParams& p, const float* coef, void* state, int fp64, float* delta,
                       int warmup);   // returns the task's block count
// positions per thread of the filter step on a device (2, 4 or 8; 4 until tuned)
int iir_positions(int dev);
bool iir_set_positions(int dev, int positions);
// times the filter at 2 / 4 / 8 positions per thread (ms[3]) and keeps the fastest
cudaError_t iir_autotune(int dev, float ms[3], int* chosen);
cudaError_t launch_iir_multi(const void* d_args, const int* d_map, unsigned blocks, int preseed,
                             cudaStream_t st);
unsigned transfer_grid(TransferParams& p, unsigned& gx, unsigned& gy);
// guided filter rows per sweep segment on a device (default 64)
int guided_rows(int dev);
bool guided_set_rows(int dev, int rows);
// times the sweep at each candidate segment height, keeps the fastest
cudaError_t guided_autotune(int dev, const int* cand, int nc, float* ms, int* chosen);
cudaError_t launch_transfer_multi(int edge_aware, const TransferParams* d_params, const int* d_map,
                                  unsigned blocks, cudaStream_t st);
// a tick's parameter table from pinned host memory (its device-mapped
// address) into device memory, read by a kernel over the host link: no copy
// engine, so it never queues behind a frame copy; bytes rounded up to 16
cudaError_t launch_table_copy(void* dst, const void* host_mapped, size_t bytes, cudaStream_t st);

}  // namespace wema
