// session.h - per-stream device state and the per-frame pipeline (host side).
#pragma once

#include <cuda_runtime.h>
#include <string>

#include "common.cuh"
#include "kernels.h"
#include "wema_cuda.h"

namespace wema {

// thread-local last-error message shared by every C entry point
void set_error(const char* fmt, ...);
void clear_error();
const char* last_error();
bool cuda_ok(cudaError_t e, const char* what);

// one-time per-device kernel attribute setup; also makes `dev` current
bool ensure_device(int dev);

// host-side IIR design, identical in arithmetic to the reference build
int design_bandpass(float f_low, float f_high, float fs, float c[10], int* warmup);
float fade_amp(float amp_factor, int frames_before, int warmup);

class Session {
public:
    wema_cuda_config cfg{};
    Geom g{};
    int nch = 1;
    IirParams ip{};
    float coef10[10] = {};
    int warmup = 0;
    int frames_processed = 0;
    int head = 0, filled = 0;          // window ring
    bool last_passthrough = false;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;       // threshold branch, joined before the inverse
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float last_alpha[3] = {};          // per-channel alpha of the last frame
    bool thr_hist = false;             // threshold scratch holds the last frame's binades

    // device arena
    void* arena = nullptr;
    size_t arena_bytes = 0;
    float* coef[3] = {};
    float* ampl[3] = {};
    float* delta[3] = {};
    float4* state[3] = {};
    float* ll[3][WEMA_MAX_LEV] = {};
    float* rec[3][WEMA_MAX_LEV] = {};  // rec[c][0]: level-0 reconstruction
    float* gray_in[3] = {};
    float* ring[3] = {};
    ThrScratch thr_s[3] = {};
    float* d_small = nullptr;          // thr[3], sum[3]
    // per-stage timing (CUDA events), enabled on demand
    enum { ST_FWD0, ST_FWD, ST_THR, ST_TEMPORAL, ST_INV, ST_XFER, N_STAGE };
    // events: 0 fwd0, 1 fwd levels, 2 temporal start, 3 temporal end, 4 inverse
    // start (after the join), 5 transfer start, 6 end, 7/8 threshold begin/end
    enum { N_EV = 9 };
    bool timing = false;
    cudaEvent_t ev[N_EV] = {};
    bool ev_pending = false;
    double stage_ms[N_STAGE] = {};
    long long stage_frames = 0;
    void mark(int k, cudaStream_t st) { if (timing) cudaEventRecord(ev[k], st); }
    bool materialize_amplified();      // ampl[] = amplified coefficients of the last frame
    bool collect_timing();
    // host-API staging (allocated on first use)
    uint8_t* stage_u8 = nullptr;       // in [3P] + out [3P]
    float* stage_f32 = nullptr;        // in [3P] + out [3P]

    ~Session();
    static size_t bytes_for(const wema_cuda_config& c);
    bool init(const wema_cuda_config& c);
    // one frame; exactly one of in_u8 / in_f32 is set; outputs optional
    bool run(const uint8_t* in_u8, const float* in_f32, uint8_t* out_u8, float* out_f32,
             cudaStream_t st);
    PyrView view(int c) const;
    bool ensure_staging();
};

}  // namespace wema
