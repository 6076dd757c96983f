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

constexpr int kSlots = 4;   // frames in flight per session (pyramid buffer sets)

// Buffers of one frame in flight
struct Slot {
    float* coef[3] = {};
    float* delta[3] = {};
    float* ll[3][WEMA_MAX_LEV] = {};
    float* rec[3][WEMA_MAX_LEV] = {};  // rec[c][0]: level-0 reconstruction (luma: gray_out)
    float* gray_in[3] = {};            // inspection only
    float* thr = nullptr;              // [0..2] thresholds, [4..6] sums
    float alpha[3] = {};
    bool valid = false;                // holds a processed frame
    bool passthrough = false;
    cudaEvent_t ev_fwd = nullptr, ev_tmp = nullptr, ev_thr = nullptr, ev_done = nullptr;
};

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
    bool inspect = false;              // keep input / reconstructed planes for reading back
    long long frames_run = 0;          // frames issued (slot = frames_run % kSlots)
    long long launches = 0;            // kernels launched by run()
    int last_slot = -1;

    // streams: forward DWT, temporal filter, threshold, inverse + output
    cudaStream_t s_fwd = nullptr, s_tmp = nullptr, s_thr = nullptr, s_inv = nullptr;
    cudaEvent_t ev_call = nullptr, ev_last = nullptr;

    void* arena = nullptr;
    size_t arena_bytes = 0;
    cudaStream_t arena_stream = nullptr;   // set: arena from the stream-ordered pool (batched)
    Slot slot[kSlots];
    float4* state[3] = {};             // IIR state (shared by the slots, updated in frame order)
    void* ring[3] = {};                // window ring (float, or __half with ring_fp16)
    float* ampl[3] = {};               // materialised amplified coefficients (inspection)
    ThrScratch thr_s[3] = {};          // threshold scratch + binade history (frame order)
    bool thr_hist = false;
    // host-API staging (allocated on first use)
    uint8_t* stage_u8 = nullptr;       // in [3P] + out [3P]
    float* stage_f32 = nullptr;        // in [3P] + out [3P]

    // per-stage timing (CUDA events on each stage's stream), enabled on demand
    enum { ST_FWD0, ST_FWD, ST_THR, ST_TEMPORAL, ST_INV, ST_INV0, ST_XFER, N_STAGE };
    enum { N_EV = 2 * N_STAGE };
    bool timing = false;
    cudaEvent_t ev[N_EV] = {};
    bool ev_pending = false;
    double stage_ms[N_STAGE] = {};
    long long stage_frames = 0;
    void mark(int k, cudaStream_t st) { if (timing) cudaEventRecord(ev[k], st); }
    bool collect_timing();

    ~Session();
    int nslots = kSlots;               // buffer sets in use (a batched stream keeps one)
    static size_t bytes_for(const wema_cuda_config& c, int nslots = kSlots);
    // alloc_stream set (a batched stream): the state comes from the device's
    // stream-ordered pool, zeroed in order on that stream, and the session
    // creates no streams or events of its own; no call synchronises the device
    bool init(const wema_cuda_config& c, int nslots = kSlots, cudaStream_t alloc_stream = nullptr);
    // One frame, asynchronous: waits for `wait` (may be null) before touching
    // in/out, records `done` (may be null) once out is written and in is no
    // longer read.  Exactly one of in_u8 / in_f32 is set; outputs optional.
    bool run(const uint8_t* in_u8, const float* in_f32, uint8_t* out_u8, float* out_f32,
             cudaEvent_t wait, cudaEvent_t done);
    // synchronous-on-a-stream form: ordered after earlier work on st; st waits for the frame
    bool run_on(const uint8_t* in_u8, const float* in_f32, uint8_t* out_u8, float* out_f32,
                cudaStream_t st);
    bool sync_all();
    // the forward transform's temporal-filter fields for level l of the frame being issued
    void fill_temporal(FwdLevelParams& p, int l) const;
    PyrView view(int b, int c) const;
    bool ensure_staging();
    bool materialize_amplified();      // ampl[] = amplified coefficients of the last frame

    // snapshot / restore of the whole stream state (the caller has waited for
    // the session's work): a header of the host-side frame counters, then the
    // device state.  Restore needs a session of the same config and buffer sets.
    size_t snapshot_bytes() const;
    bool snapshot(void* host, size_t cap) const;
    bool restore(const void* host, size_t bytes);
};

}  // namespace wema
