// session.cu - per-stream pipeline and the wema_cuda_* entry points.
//
// A Session owns every device buffer of one video stream in a single
// allocation: the unique detail planes (orig, amplified, deltas), the IIR
// state (float4 per coefficient) or the window ring, the LL / reconstruction
// planes of each level, the threshold scratch and a few scalars.  A frame is
// a fixed sequence of launches on one stream:
//   forward DWT (L launches, level 0 reads RGB and converts on the fly)
//   exact threshold (2 launches for all channels; 4 on the first frame)
//   [first frame: preseed]  IIR + amplify  |  ring push + window amplify
//   inverse DWT (L launches; colour writes RGB at level 0)
//   luma: guided filter / Gaussian + RGB transfer + u8 quantisation
// mirroring wema_process_frame (wema.c:746-952).
#include "session.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <new>
#include <vector>

namespace wema {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
void clear_error() { g_err.clear(); }
const char* last_error() { return g_err.c_str(); }

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return false;
}

bool ensure_device(int dev) {
    static std::mutex mu;
    static std::vector<char> ready;
    if (!cuda_ok(cudaSetDevice(dev), "cudaSetDevice")) return false;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)ready.size() <= dev) ready.resize(dev + 1, 0);
    if (ready[dev]) return true;
    if (!cuda_ok(dwt_prepare_device(), "DWT kernel setup")) return false;
    if (!cuda_ok(spatial_prepare_device(), "spatial kernel setup")) return false;
    if (!cuda_ok(thr_prepare_device(), "threshold kernel setup")) return false;
    ready[dev] = 1;
    return true;
}

// ---------------------------------------------------------------- IIR design
#define WEMA_PI_F ((float)3.14159265358979323846)

// iir_design_bandpass / iir_temporal_init (iir_filter.c:36-154), evaluated
// the way the reference's -Ofast build evaluates it (FMA placement read
// from GCC's optimised-tree dump of that build).
int design_bandpass(float f_low, float f_high, float fs, float c[10], int* warmup) {
    if (f_low >= f_high || f_low <= 0 || fs * 0.5f <= f_high) return -1;
    const float s2 = 1.41421356237f;
    float wc = tanf((f_low * WEMA_PI_F) / fs);
    float ws2 = wc * s2;
    float norm = 1.0f / (fmaf(wc, wc, ws2) + 1.0f);
    c[0] = norm;
    c[1] = norm * -2.0f;
    c[2] = norm;
    c[3] = (fmaf(wc, wc, -1.0f) * 2.0f) * norm;
    c[4] = (fmaf(wc, wc, 1.0f) - ws2) * norm;
    wc = tanf((f_high * WEMA_PI_F) / fs);
    float wc2 = wc * wc;
    norm = 1.0f / (fmaf(wc, s2, wc2) + 1.0f);
    c[5] = wc2 * norm;
    c[6] = c[5] * 2.0f;
    c[7] = c[5];
    c[8] = ((wc2 - 1.0f) * 2.0f) * norm;
    c[9] = norm * fmaf(-wc, s2, wc2 + 1.0f);
    if (warmup) {
        int w = (int)(7.0f * fs / (2.0f * WEMA_PI_F * f_low));
        *warmup = w < 30 ? 30 : w;
    }
    return 0;
}

// quadratic 15-frame fade-in after the preseed (wema.c:831-839)
float fade_amp(float amp_factor, int frames_before, int warmup) {
    const int g = frames_before - warmup;
    if (g < 0) return 0.0f;
    if (g >= 15) return amp_factor;
    const float t = (float)(g + 1) * (1.0f / 15.0f);
    return (t * t) * amp_factor;
}

// ------------------------------------------------------------------- arena

namespace {
struct Arena {
    size_t off = 0;
    char* base = nullptr;
    template <class T>
    T* take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T* p = base ? (T*)(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
};
}  // namespace

static void layout(Arena& A, Session& s) {
    const Geom& g = s.g;
    const long long pu = g.uoff[g.levels];
    const long long n6 = g.off6[g.levels];
    for (int b = 0; b < s.nslots; b++) {
        Slot& q = s.slot[b];
        // planes_fp16: coefficient and delta planes and the level-0 reconstruction
        // (the frame) in FP16 (float* kept); the LL and coarser reconstructions
        // stay FP32 - their values grow about 2x per level, so FP16 there would
        // quantise the coarse bands far more coarsely than the frame
        auto plane = [&](long long n, bool h) {
            return h ? reinterpret_cast<float*>(A.take<uint16_t>(n)) : A.take<float>(n);
        };
        const bool h = s.cfg.planes_fp16;
        for (int c = 0; c < s.nch; c++) {
            q.coef[c] = plane(pu, h);
            q.delta[c] = plane(pu, h);
            for (int l = 0; l < g.levels; l++) q.ll[c][l] = plane(g.n[l], false);
            for (int l = 0; l < g.levels; l++) q.rec[c][l] = plane((long long)g.in_w[l] * g.in_h[l], h && l == 0);
            q.gray_in[c] = A.take<float>(g.pixels);
        }
        q.thr = A.take<float>(8);
    }
    for (int c = 0; c < s.nch; c++) {
        if (s.cfg.use_iir) s.state[c] = A.take<float4>(s.cfg.iir_state_fp64 ? 2 * pu : pu);
        else if (s.cfg.ring_fp16) s.ring[c] = A.take<uint16_t>((size_t)pu * s.cfg.temporal_window);
        else s.ring[c] = A.take<float>((size_t)pu * s.cfg.temporal_window);
        s.ampl[c] = A.take<float>(pu);
        void* t = A.take<char>(thr_scratch_bytes(n6));
        if (A.base) thr_scratch_bind(s.thr_s[c], t, n6);
    }
}

static bool valid_config(const wema_cuda_config& c) {
    if (c.width < 1 || c.height < 1) { set_error("frame size must be positive"); return false; }
    if ((long long)c.width * c.height > (1LL << 28)) { set_error("frame too large"); return false; }
    if (!(c.fps > 0)) { set_error("fps must be positive"); return false; }
    if (!c.use_iir && (c.temporal_window < 4 || c.temporal_window > 256)) {
        set_error("temporal window must be in [4, 256]");
        return false;
    }
    if (c.iir_state_fp64 != 0 && c.iir_state_fp64 != 1) { set_error("iir_state_fp64 must be 0 or 1"); return false; }
    if (c.ring_fp16 != 0 && c.ring_fp16 != 1) { set_error("ring_fp16 must be 0 or 1"); return false; }
    if (c.planes_fp16 != 0 && c.planes_fp16 != 1) { set_error("planes_fp16 must be 0 or 1"); return false; }
    return true;
}

size_t Session::bytes_for(const wema_cuda_config& c, int nslots) {
    if (!valid_config(c)) return 0;
    Session s;
    s.nslots = nslots < 1 ? 1 : (nslots > kSlots ? kSlots : nslots);
    s.cfg = c;
    s.g = make_geom(c.width, c.height);
    s.nch = c.color_mode ? 3 : 1;
    Arena A;
    layout(A, s);
    return A.off;
}

Session::~Session() {
    for (cudaStream_t st : {s_fwd, s_tmp, s_thr, s_inv})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    for (Slot& q : slot)
        for (cudaEvent_t e : {q.ev_fwd, q.ev_tmp, q.ev_thr, q.ev_done})
            if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_call, ev_last})
        if (e) cudaEventDestroy(e);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (arena && arena_stream) cudaFreeAsync(arena, arena_stream);
    else if (arena) cudaFree(arena);
    if (stage_u8) cudaFree(stage_u8);
    if (stage_f32) cudaFree(stage_f32);
}

// adds the last timed frame's per-stage durations (waits for it)
bool Session::collect_timing() {
    if (!ev_pending) return true;
    ev_pending = false;
    for (int k = 0; k < N_STAGE; k++) {
        if (!cuda_ok(cudaEventSynchronize(ev[2 * k + 1]), "event sync")) return false;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]) == cudaSuccess) stage_ms[k] += ms;
    }
    stage_frames++;
    return true;
}

bool Session::init(const wema_cuda_config& c, int ns, cudaStream_t alloc_stream) {
    if (!valid_config(c)) return false;
    nslots = ns < 1 ? 1 : (ns > kSlots ? kSlots : ns);
    cfg = c;
    if (!ensure_device(c.device)) return false;
    g = make_geom(c.width, c.height);
    nch = c.color_mode ? 3 : 1;
    if (c.use_iir) {
        if (design_bandpass(c.f_low, c.f_high, c.fps, coef10, &warmup) < 0) {
            set_error("invalid band: need 0 < f_low < f_high < fps/2 (iir_filter.c:74)");
            return false;
        }
    }
    memcpy(ip.c, coef10, sizeof coef10);
    ip.levels = g.levels;
    for (int l = 0; l <= g.levels; l++) { ip.uoff[l] = g.uoff[l]; ip.off6[l] = g.off6[l]; }
    for (int l = 0; l < g.levels; l++) ip.n[l] = g.n[l];
    ip.simd_end = g.off6[g.levels] & ~15LL;
    ip.h16 = c.planes_fp16;

    Arena A;
    layout(A, *this);
    arena_bytes = A.off;
    if (alloc_stream) {
        if (!cuda_ok(cudaMallocAsync(&arena, arena_bytes, alloc_stream), "cudaMallocAsync(session)"))
            return false;
        arena_stream = alloc_stream;
        if (!cuda_ok(cudaMemsetAsync(arena, 0, arena_bytes, alloc_stream), "cudaMemsetAsync")) return false;
        A = Arena();
        A.base = (char*)arena;
        layout(A, *this);
        return true;
    }
    if (!cuda_ok(cudaMalloc(&arena, arena_bytes), "cudaMalloc(session)")) return false;
    if (!cuda_ok(cudaMemset(arena, 0, arena_bytes), "cudaMemset")) return false;
    A = Arena();
    A.base = (char*)arena;
    layout(A, *this);
    for (cudaStream_t* st : {&s_fwd, &s_tmp, &s_thr, &s_inv})
        if (!cuda_ok(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "cudaStreamCreate"))
            return false;
    for (Slot& q : slot)
        for (cudaEvent_t* e : {&q.ev_fwd, &q.ev_tmp, &q.ev_thr, &q.ev_done})
            if (!cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate"))
                return false;
    for (cudaEvent_t* e : {&ev_call, &ev_last})
        if (!cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate"))
            return false;
    return true;
}

bool Session::sync_all() {
    for (cudaStream_t st : {s_fwd, s_tmp, s_thr, s_inv})
        if (!cuda_ok(cudaStreamSynchronize(st), "sync")) return false;
    return true;
}

bool Session::materialize_amplified() {
    if (last_slot < 0) { set_error("no frame processed yet"); return false; }
    const Slot& q = slot[last_slot];
    if (!sync_all()) return false;
    for (int c = 0; c < nch; c++)
        if (!cuda_ok(launch_amplify(ip, q.coef[c], q.delta[c], q.thr + c, q.alpha[c], ampl[c], s_inv),
                     "amplify"))
            return false;
    return cuda_ok(cudaStreamSynchronize(s_inv), "sync");
}

bool Session::ensure_staging() {
    if (stage_u8) return true;
    const size_t P3 = 3 * (size_t)g.pixels;
    if (!cuda_ok(cudaMalloc(&stage_u8, 2 * P3), "cudaMalloc(staging)")) return false;
    if (!cuda_ok(cudaMalloc(&stage_f32, 2 * P3 * sizeof(float)), "cudaMalloc(staging)")) return false;
    return true;
}

PyrView Session::view(int b, int c) const {
    PyrView v{};
    v.coef = slot[b].coef[c];
    v.levels = g.levels;
    for (int l = 0; l < g.levels; l++) { v.n[l] = g.n[l]; v.uoff[l] = g.uoff[l]; }
    for (int l = 0; l <= g.levels; l++) v.off6[l] = g.off6[l];
    return v;
}

// The forward transform's parameters for running the filter's step on level
// l's coefficients of the current slot (state, deltas, coefficients, tail
// bound): a batched stream after its first frame (Batch::tick).
void Session::fill_temporal(FwdLevelParams& p, int l) const {
    const Slot& q = slot[(int)(frames_run % nslots)];
    memcpy(p.iir_c, coef10, sizeof coef10);
    p.iir_off6 = g.off6[l];
    p.iir_simd_end = ip.simd_end;
    p.iir_fp64 = cfg.iir_state_fp64;
    for (int c = 0; c < nch; c++) {
        p.iir_state[c] = cfg.iir_state_fp64 ? (void*)(reinterpret_cast<double2*>(state[c]) + 2 * g.uoff[l])
                                            : (void*)(state[c] + g.uoff[l]);
        p.iir_delta[c] = plane_at(q.delta[c], g.uoff[l], cfg.planes_fp16);
    }
}

// Frame pipeline.  Each frame uses one of kSlots buffer sets and four
// streams: forward DWT -> {temporal filter, threshold} -> inverse + output,
// chained by the slot's events.  The temporal filter and the threshold run in
// frame order on their own streams (IIR state, window ring and binade history
// carry from frame to frame), and frame t+1's forward DWT and filter overlap
// frame t's threshold and inverse.
bool Session::run(const uint8_t* in_u8, const float* in_f32, uint8_t* out_u8, float* out_f32,
                  cudaEvent_t wait, cudaEvent_t done) {
    const int L = g.levels;
    const int b = (int)(frames_run % nslots);
    Slot& q = slot[b];
    if (timing) {
        if (!collect_timing()) return false;
        if (!ev[0])
            for (auto& e : ev)
                if (!cuda_ok(cudaEventCreate(&e), "cudaEventCreate")) return false;
    }
    // the slot's previous frame must have finished with its buffers
    if (wait && !cuda_ok(cudaStreamWaitEvent(s_fwd, wait, 0), "stream wait")) return false;
    if (q.valid && !cuda_ok(cudaStreamWaitEvent(s_fwd, q.ev_done, 0), "stream wait")) return false;

    // ---- forward DWT
    mark(2 * ST_FWD0, s_fwd);
    for (int l = 0; l < L; l++) {
        FwdLevelParams p{};
        p.iw = g.in_w[l];
        p.ih = g.in_h[l];
        p.sw = g.sw[l];
        p.sh = g.sh[l];
        p.n = g.n[l];
        p.vec_end = vec_cover(g.pixels);
        int mode = kSrcPlanes;
        if (l == 0) {
            mode = in_u8 ? kSrcRgbU8 : kSrcRgbF32;
            p.src_u8 = in_u8;
            p.src_f32 = in_f32;
            if (inspect)
                for (int c = 0; c < nch; c++) p.plane_out[c] = q.gray_in[c];
        } else {
            for (int c = 0; c < nch; c++) p.src_planes[c] = q.ll[c][l - 1];
        }
        const bool h = cfg.planes_fp16;
        for (int c = 0; c < nch; c++) {
            p.coef[c] = plane_at(q.coef[c], g.uoff[l], h);
            p.prev[c] = l > 0 ? plane_at(q.coef[c], g.uoff[l - 1], h) : nullptr;
            p.ll_out[c] = q.ll[c][l];
        }
        p.prev_n = l > 0 ? g.n[l - 1] : 0;
        p.h16 = h;
        if (!cuda_ok(launch_dwt_fwd(mode, nch, p, s_fwd), "forward DWT")) return false;
        launches++;
        if (l == 0) {
            mark(2 * ST_FWD0 + 1, s_fwd);
            mark(2 * ST_FWD, s_fwd);
        }
    }
    mark(2 * ST_FWD + 1, s_fwd);
    if (!cuda_ok(cudaEventRecord(q.ev_fwd, s_fwd), "event record")) return false;

    // ---- temporal filter (frame order on s_tmp)
    if (!cuda_ok(cudaStreamWaitEvent(s_tmp, q.ev_fwd, 0), "stream wait")) return false;
    const long long pu = g.uoff[L];
    q.passthrough = false;
    mark(2 * ST_TEMPORAL, s_tmp);
    if (cfg.use_iir) {
        if (frames_processed == 0) {   // iir_temporal_preseed on the first frame
            for (int c = 0; c < nch; c++)
                if (!cuda_ok(launch_iir_preseed(ip, q.coef[c], state[c], cfg.iir_state_fp64, warmup, s_tmp), "preseed"))
                    return false;
            launches += nch;
            frames_processed = warmup;
        }
        const float amp = fade_amp(cfg.amp_factor, frames_processed, warmup);
        frames_processed++;
        q.alpha[0] = amp;
        q.alpha[1] = q.alpha[2] = amp * 0.5f;
        // (a batched stream runs this step inside its forward transform after
        // its first frame, Batch::tick; here the filter is its own launch on
        // s_tmp, beside the threshold - the shorter latency for a frame that
        // is waited for)
        for (int c = 0; c < nch; c++)
            if (!cuda_ok(launch_iir(ip, q.coef[c], state[c], cfg.iir_state_fp64, q.delta[c], s_tmp), "IIR"))
                return false;
        launches += nch;
    } else {
        for (int c = 0; c < nch; c++)
            if (!cuda_ok(launch_ring_push(q.coef[c], cfg.planes_fp16, ring[c], cfg.ring_fp16, pu, head, s_tmp),
                         "ring push"))
                return false;
        launches += nch;
        head = (head + 1) % cfg.temporal_window;
        if (filled < cfg.temporal_window) filled++;
        q.passthrough = filled < cfg.temporal_window;   // wema.c:924-929
        q.alpha[0] = cfg.amp_factor;
        q.alpha[1] = q.alpha[2] = cfg.amp_factor * 0.5f;
        if (!q.passthrough) {
            WindowParams wp{};
            wp.pu = pu;
            wp.ws = cfg.temporal_window;
            wp.head = head;   // oldest sample (temporal_filter.c:221)
            wp.bilateral = cfg.bilateral_temp;
            wp.fp16 = cfg.ring_fp16;
            wp.h16 = cfg.planes_fp16;
            const int ws = cfg.temporal_window, center = ws / 2;
            const float ts = (float)ws * 0.15f;
            const float inv2 = 0.5f / (ts * ts);
            for (int t = 0; t < ws; t++) {
                const float d = (float)(t - center);
                wp.time_w[t] = expf(-(d * d) * inv2);
            }
            for (int c = 0; c < nch; c++)
                if (!cuda_ok(launch_window(wp, ring[c], q.delta[c], s_tmp), "window filter"))
                    return false;
            launches += nch;
        }
    }
    mark(2 * ST_TEMPORAL + 1, s_tmp);
    if (!cuda_ok(cudaEventRecord(q.ev_tmp, s_tmp), "event record")) return false;

    // ---- threshold (frame order on s_thr: the binade history carries over)
    if (!q.passthrough) {
        if (!cuda_ok(cudaStreamWaitEvent(s_thr, q.ev_fwd, 0), "stream wait")) return false;
        PyrView views[3];
        for (int c = 0; c < nch; c++) views[c] = view(b, c);
        ThrScratch ts[3];
        for (int c = 0; c < nch; c++) ts[c] = thr_s[c];
        mark(2 * ST_THR, s_thr);
        if (!cuda_ok(launch_threshold(views, nch, ts, q.thr, q.thr + 4, cfg.threshold_form,
                                      thr_hist ? 1 : 0, cfg.planes_fp16, s_thr),
                     "threshold"))
            return false;
        // monoids + walk; partial sums + prefix without history; one launch over FP16 planes
        launches += cfg.planes_fp16 ? 1 : (thr_hist ? 2 : 4);
        thr_hist = true;
        mark(2 * ST_THR + 1, s_thr);
        if (!cuda_ok(cudaEventRecord(q.ev_thr, s_thr), "event record")) return false;
    }

    // ---- inverse DWT (amplification applied while staging) and output
    if (!cuda_ok(cudaStreamWaitEvent(s_inv, q.ev_tmp, 0), "stream wait")) return false;
    if (!q.passthrough && !cuda_ok(cudaStreamWaitEvent(s_inv, q.ev_thr, 0), "stream wait"))
        return false;
    if (q.passthrough) {
        TransferParams tp{};
        tp.w = g.w;
        tp.h = g.h;
        tp.src_u8 = in_u8;
        tp.src_f32 = in_f32;
        tp.out_u8 = out_u8;
        tp.out_f32 = out_f32;
        if (!cuda_ok(launch_passthrough(tp, s_inv), "passthrough")) return false;
        launches++;
    } else {
        mark(2 * ST_INV, s_inv);
        for (int l = L - 1; l >= 0; l--) {
            InvLevelParams iq{};
            iq.ow = g.in_w[l];
            iq.oh = g.in_h[l];
            iq.sw = g.sw[l];
            iq.sh = g.sh[l];
            iq.n = g.n[l];
            iq.thr = q.thr;
            const bool h = cfg.planes_fp16;
            iq.h16 = h;
            iq.out16 = h && l == 0;
            for (int c = 0; c < nch; c++) {
                iq.ll[c] = (l == L - 1) ? q.ll[c][L - 1] : q.rec[c][l + 1];
                iq.coef[c] = plane_at(q.coef[c], g.uoff[l], h);
                iq.delta[c] = plane_at(q.delta[c], g.uoff[l], h);
                iq.alpha[c] = l == 0 ? q.alpha[c] * 0.5f : q.alpha[c];
                iq.out_planes[c] = (l > 0 || nch == 1 || inspect) ? q.rec[c][l] : nullptr;
            }
            if (l == 0) {
                mark(2 * ST_INV + 1, s_inv);
                mark(2 * ST_INV0, s_inv);
            }
            int mode = kOutPlanes;
            if (l == 0 && nch == 3) {
                mode = kOutRgb;
                iq.out_u8 = out_u8;
                iq.out_f32 = out_f32;
            }
            if (!cuda_ok(launch_dwt_inv(nch, mode, iq, s_inv), "inverse DWT")) return false;
            launches++;
        }
        mark(2 * ST_INV0 + 1, s_inv);
        mark(2 * ST_XFER, s_inv);
        if (nch == 1) {
            TransferParams tp{};
            tp.w = g.w;
            tp.h = g.h;
            tp.vec_end = vec_cover(g.pixels);
            tp.src_u8 = in_u8;
            tp.src_f32 = in_f32;
            tp.gray_out = q.rec[0][0];
            tp.out_u8 = out_u8;
            tp.out_f32 = out_f32;
            tp.edge_aware = cfg.edge_aware;
            tp.h16 = cfg.planes_fp16;
            if (!cuda_ok(launch_transfer(tp, s_inv), "luma transfer")) return false;
            launches++;
        }
        mark(2 * ST_XFER + 1, s_inv);
        ev_pending = timing;
    }
    if (!cuda_ok(cudaEventRecord(q.ev_done, s_inv), "event record")) return false;
    if (done && !cuda_ok(cudaEventRecord(done, s_inv), "event record")) return false;
    q.valid = true;
    last_slot = b;
    frames_run++;
    return true;
}

bool Session::run_on(const uint8_t* in_u8, const float* in_f32, uint8_t* out_u8, float* out_f32,
                     cudaStream_t st) {
    if (!cuda_ok(cudaEventRecord(ev_call, st), "event record")) return false;
    if (!run(in_u8, in_f32, out_u8, out_f32, ev_call, ev_last)) return false;
    return cuda_ok(cudaStreamWaitEvent(st, ev_last, 0), "stream wait");
}

}  // namespace wema

// ===================================================================== C ABI
using namespace wema;

// ---------------------------------------------------------------- snapshot
namespace {
struct SnapHeader {
    char magic[8];                     // "WEMASNAP"
    int version, nslots;
    wema_cuda_config cfg;
    unsigned long long arena_bytes;
    long long frames_run;
    int frames_processed, head, filled, last_slot, thr_hist;
    int valid[kSlots], passthrough[kSlots];
    float alpha[kSlots][3];
};
constexpr int kSnapVersion = 1;
}  // namespace

size_t Session::snapshot_bytes() const { return sizeof(SnapHeader) + arena_bytes; }

bool Session::snapshot(void* host, size_t cap) const {
    if (!host || cap < snapshot_bytes()) { set_error("snapshot needs %zu bytes", snapshot_bytes()); return false; }
    SnapHeader h{};
    memcpy(h.magic, "WEMASNAP", 8);
    h.version = kSnapVersion;
    h.nslots = nslots;
    h.cfg = cfg;
    h.arena_bytes = arena_bytes;
    h.frames_run = frames_run;
    h.frames_processed = frames_processed;
    h.head = head;
    h.filled = filled;
    h.last_slot = last_slot;
    h.thr_hist = thr_hist;
    for (int i = 0; i < kSlots; i++) {
        h.valid[i] = slot[i].valid;
        h.passthrough[i] = slot[i].passthrough;
        for (int c = 0; c < 3; c++) h.alpha[i][c] = slot[i].alpha[c];
    }
    memcpy(host, &h, sizeof h);
    return cuda_ok(cudaMemcpy((char*)host + sizeof h, arena, arena_bytes, cudaMemcpyDeviceToHost),
                   "snapshot copy");
}

bool Session::restore(const void* host, size_t bytes) {
    SnapHeader h;
    if (!host || bytes < sizeof h) { set_error("not a session snapshot"); return false; }
    memcpy(&h, host, sizeof h);
    if (memcmp(h.magic, "WEMASNAP", 8) || h.version != kSnapVersion) {
        set_error("not a session snapshot (or another version)");
        return false;
    }
    wema_cuda_config a = h.cfg, b = cfg;
    a.device = b.device = 0;             // a snapshot may move to another device
    if (memcmp(&a, &b, sizeof a) || h.nslots != nslots || h.arena_bytes != arena_bytes ||
        bytes < sizeof h + arena_bytes) {
        set_error("snapshot is of another stream configuration");
        return false;
    }
    // from pageable memory cudaMemcpy may return before its DMA lands, and the
    // session's streams are non-blocking (not ordered after the legacy
    // stream): wait for the legacy stream before the next frame can read
    if (!cuda_ok(cudaMemcpy(arena, (const char*)host + sizeof h, arena_bytes, cudaMemcpyHostToDevice),
                 "restore copy") ||
        !cuda_ok(cudaStreamSynchronize(cudaStreamLegacy), "restore copy sync"))
        return false;
    frames_run = h.frames_run;
    frames_processed = h.frames_processed;
    head = h.head;
    filled = h.filled;
    last_slot = h.last_slot;
    thr_hist = h.thr_hist != 0;
    for (int i = 0; i < kSlots; i++) {
        slot[i].valid = h.valid[i] != 0;
        slot[i].passthrough = h.passthrough[i] != 0;
        for (int c = 0; c < 3; c++) slot[i].alpha[c] = h.alpha[i][c];
    }
    return true;
}

// IEEE binary16 bits -> float (exact)
static float half_bits_to_float(uint16_t h) {
    const uint32_t sgn = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu, bits;
    if (e == 0x1f) bits = sgn | 0x7f800000u | (m << 13);                  // inf / nan
    else if (e) bits = sgn | ((e + 112u) << 23) | (m << 13);              // normal
    else if (!m) bits = sgn;                                              // zero
    else {                                                                // subnormal: renormalise
        int sh = 0;
        while (!(m & 0x400u)) { m <<= 1; sh++; }
        bits = sgn | ((uint32_t)(113 - sh) << 23) | ((m & 0x3ffu) << 13);
    }
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
}

struct wema_cuda_session {
    Session s;
};

#define WEMA_API extern "C" __attribute__((visibility("default")))

WEMA_API const char* wema_cuda_last_error(void) { return last_error(); }

WEMA_API void wema_cuda_config_default(wema_cuda_config* cfg, int width, int height, float fps) {
    memset(cfg, 0, sizeof *cfg);
    cfg->width = width;
    cfg->height = height;
    cfg->fps = fps;
    cfg->amp_factor = 120.0f;
    cfg->f_low = 0.5f;
    cfg->f_high = fps / 2.0f - 0.0001f;   // main.c:248-250
    cfg->temporal_window = 32;
    cfg->edge_aware = 1;
    cfg->bilateral_temp = 0;
    cfg->color_mode = 0;
    cfg->use_iir = 1;
    cfg->threshold_form = WEMA_CUDA_THR_SINGLE;
    cfg->device = 0;
}

WEMA_API size_t wema_cuda_session_bytes(const wema_cuda_config* cfg) {
    clear_error();
    if (!cfg) { set_error("null config"); return 0; }
    return Session::bytes_for(*cfg);
}

WEMA_API int wema_cuda_session_create(const wema_cuda_config* cfg, wema_cuda_session** out) {
    clear_error();
    if (!cfg || !out) { set_error("null argument"); return -1; }
    *out = nullptr;
    wema_cuda_session* s = new (std::nothrow) wema_cuda_session();
    if (!s) { set_error("out of host memory"); return -1; }
    if (!s->s.init(*cfg)) {
        delete s;
        return -1;
    }
    *out = s;
    return 0;
}

WEMA_API void wema_cuda_session_destroy(wema_cuda_session* s) {
    if (!s) return;
    cudaSetDevice(s->s.cfg.device);
    delete s;
}

WEMA_API int wema_cuda_process_u8(wema_cuda_session* s, const uint8_t* d_in, uint8_t* d_out,
                                  void* cuda_stream) {
    clear_error();
    if (!s || !d_in || !d_out) { set_error("null argument"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice")) return -1;
    if (!cuda_stream) return s->s.run(d_in, nullptr, d_out, nullptr, nullptr, nullptr) ? 0 : -1;
    return s->s.run_on(d_in, nullptr, d_out, nullptr, (cudaStream_t)cuda_stream) ? 0 : -1;
}

WEMA_API int wema_cuda_process_u8_async(wema_cuda_session* s, const uint8_t* d_in, uint8_t* d_out,
                                        void* wait_event, void* done_event) {
    clear_error();
    if (!s || !d_in || !d_out) { set_error("null argument"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice")) return -1;
    return s->s.run(d_in, nullptr, d_out, nullptr, (cudaEvent_t)wait_event, (cudaEvent_t)done_event)
               ? 0 : -1;
}

WEMA_API int wema_cuda_process_f32(wema_cuda_session* s, const float* d_in, float* d_out_f32,
                                   uint8_t* d_out_u8, void* cuda_stream) {
    clear_error();
    if (!s || !d_in || (!d_out_f32 && !d_out_u8)) { set_error("null argument"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice")) return -1;
    if (!cuda_stream) return s->s.run(nullptr, d_in, d_out_u8, d_out_f32, nullptr, nullptr) ? 0 : -1;
    return s->s.run_on(nullptr, d_in, d_out_u8, d_out_f32, (cudaStream_t)cuda_stream) ? 0 : -1;
}

WEMA_API int wema_cuda_process_host_u8(wema_cuda_session* s, const uint8_t* h_in, uint8_t* h_out) {
    clear_error();
    if (!s || !h_in || !h_out) { set_error("null argument"); return -1; }
    Session& S = s->s;
    if (!cuda_ok(cudaSetDevice(S.cfg.device), "cudaSetDevice")) return -1;
    if (!S.ensure_staging()) return -1;
    const size_t P3 = 3 * (size_t)S.g.pixels;
    // the staging buffers are reused: everything earlier on this session has finished
    if (!S.sync_all()) return -1;
    if (!cuda_ok(cudaMemcpyAsync(S.stage_u8, h_in, P3, cudaMemcpyHostToDevice, S.s_fwd), "H2D"))
        return -1;
    if (!S.run(S.stage_u8, nullptr, S.stage_u8 + P3, nullptr, nullptr, nullptr)) return -1;
    if (!cuda_ok(cudaMemcpyAsync(h_out, S.stage_u8 + P3, P3, cudaMemcpyDeviceToHost, S.s_inv), "D2H"))
        return -1;
    return cuda_ok(cudaStreamSynchronize(S.s_inv), "sync") ? 0 : -1;
}

WEMA_API int wema_cuda_session_sync(wema_cuda_session* s) {
    clear_error();
    if (!s) { set_error("null session"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice")) return -1;
    return s->s.sync_all() ? 0 : -1;
}

WEMA_API int wema_cuda_autotune(int device, char* report, size_t cap) {
    clear_error();
    if (!ensure_device(device)) return -1;
    float ms[3] = {0.f, 0.f, 0.f}, gms[3] = {0.f, 0.f, 0.f}, fms[9] = {}, ims[9] = {};
    const int rows[3] = {64, 128, 256};
    int chosen = 0, grows = 0, fbest = 0, ibest = 0;
    if (!cuda_ok(iir_autotune(device, ms, &chosen), "autotune")) return -1;
    if (!cuda_ok(guided_autotune(device, rows, 3, gms, &grows), "autotune")) return -1;
    if (!cuda_ok(dwt_autotune(device, fms, ims, &fbest, &ibest), "autotune")) return -1;
    if (report && cap) {
        int n = snprintf(report, cap,
                         "iir positions per thread: 2 %.4f ms, 4 %.4f ms, 8 %.4f ms -> %d; "
                         "guided sweep rows per segment: 64 %.4f ms, 128 %.4f ms, 256 %.4f ms -> %d",
                         ms[0], ms[1], ms[2], chosen, gms[0], gms[1], gms[2], grows);
        for (int inv = 0; inv < 2 && n > 0 && (size_t)n < cap; inv++) {
            const float* t = inv ? ims : fms;
            n += snprintf(report + n, cap - n, "; %s DWT level 0 (CTAs/SM x lines/warp):",
                          inv ? "inverse" : "forward");
            for (int v = 0; v < 9 && n > 0 && (size_t)n < cap; v++) {
                int mb, lp;
                dwt_variant_shape(v, &mb, &lp);
                n += snprintf(report + n, cap - n, " %dx%d %.4f", mb, lp, t[v]);
            }
            if (n > 0 && (size_t)n < cap) {
                int mb, lp;
                dwt_variant_shape(inv ? ibest : fbest, &mb, &lp);
                n += snprintf(report + n, cap - n, " ms -> %dx%d", mb, lp);
            }
        }
    }
    return chosen;
}

WEMA_API int wema_cuda_set_guided_rows(int device, int rows) {
    clear_error();
    if (!guided_set_rows(device, rows)) {
        set_error("rows per segment must be a multiple of 16 in 16..4096");
        return -1;
    }
    return 0;
}

WEMA_API int wema_cuda_get_guided_rows(int device) {
    clear_error();
    return guided_rows(device);
}

WEMA_API int wema_cuda_set_dwt_variant(int device, int inverse, int variant) {
    clear_error();
    if (!dwt_set_variant(device, inverse, variant)) {
        set_error("DWT variant must be 0..8");
        return -1;
    }
    return 0;
}

WEMA_API int wema_cuda_get_dwt_variant(int device, int inverse) {
    clear_error();
    return dwt_variant(device, inverse);
}

WEMA_API int wema_cuda_set_iir_positions(int device, int positions) {
    clear_error();
    if (!iir_set_positions(device, positions)) { set_error("positions per thread must be 2, 4 or 8"); return -1; }
    return 0;
}

WEMA_API int wema_cuda_get_iir_positions(int device) {
    clear_error();
    return iir_positions(device);
}

WEMA_API size_t wema_cuda_session_snapshot_bytes(wema_cuda_session* s) {
    clear_error();
    if (!s) { set_error("null session"); return 0; }
    return s->s.snapshot_bytes();
}

WEMA_API int wema_cuda_session_snapshot(wema_cuda_session* s, void* host, size_t cap) {
    clear_error();
    if (!s) { set_error("null session"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice") || !s->s.sync_all()) return -1;
    return s->s.snapshot(host, cap) ? 0 : -1;
}

WEMA_API int wema_cuda_session_restore(wema_cuda_session* s, const void* host, size_t bytes) {
    clear_error();
    if (!s) { set_error("null session"); return -1; }
    if (!cuda_ok(cudaSetDevice(s->s.cfg.device), "cudaSetDevice") || !s->s.sync_all()) return -1;
    return s->s.restore(host, bytes) ? 0 : -1;
}

WEMA_API int wema_cuda_set_inspect(wema_cuda_session* s, int enable) {
    clear_error();
    if (!s) { set_error("null session"); return -1; }
    s->s.inspect = enable != 0;
    return 0;
}

WEMA_API int wema_cuda_session_frames_processed(const wema_cuda_session* s) {
    return s ? s->s.frames_processed : -1;
}

WEMA_API long wema_cuda_session_read(wema_cuda_session* s, int what, int channel, float* h_dst,
                                     size_t cap) {
    clear_error();
    if (!s || !h_dst) { set_error("null argument"); return -1; }
    Session& S = s->s;
    if (channel < 0 || channel >= S.nch) { set_error("bad channel"); return -1; }
    if (S.last_slot < 0) { set_error("no frame processed yet"); return -1; }
    if (!cuda_ok(cudaSetDevice(S.cfg.device), "cudaSetDevice")) return -1;
    if (!S.sync_all()) return -1;
    const Geom& g = S.g;
    const Slot& q = S.slot[S.last_slot];
    const long long pu = g.uoff[g.levels], n6 = g.off6[g.levels];
    // a device plane into host floats (FP16 pyramid planes converted exactly)
    auto fetch = [&](float* dst, const float* src, size_t n, bool h) -> bool {
        if (!h) return cuda_ok(cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
        std::vector<uint16_t> b(n);
        if (!cuda_ok(cudaMemcpy(b.data(), src, n * sizeof(uint16_t), cudaMemcpyDeviceToHost), "D2H"))
            return false;
        for (size_t i = 0; i < n; i++) dst[i] = half_bits_to_float(b[i]);
        return true;
    };
    const bool h16 = S.cfg.planes_fp16;
    auto rd = [&](const float* src, size_t n, bool h) -> long {
        if (n > cap) { set_error("buffer too small (%zu needed)", n); return -1; }
        return fetch(h_dst, src, n, h) ? (long)n : -1;
    };
    auto rd6 = [&](const float* src, bool h) -> long {
        if ((size_t)n6 > cap) { set_error("buffer too small (%lld needed)", n6); return -1; }
        std::vector<float> u(pu);
        if (!fetch(u.data(), src, pu, h)) return -1;
        for (int l = 0; l < g.levels; l++)
            for (int slot = 0; slot < 6; slot++) {
                const int band = slot < 3 ? slot : 5 - slot;
                memcpy(h_dst + g.off6[l] + slot * g.n[l], u.data() + g.uoff[l] + band * g.n[l],
                       g.n[l] * sizeof(float));
            }
        return (long)n6;
    };
    const bool planes = S.inspect || (what == WEMA_CUDA_READ_GRAY_OUT && S.nch == 1);
    switch (what) {
        case WEMA_CUDA_READ_GRAY_IN:
        case WEMA_CUDA_READ_GRAY_OUT:
            if (!planes) { set_error("enable wema_cuda_set_inspect before processing"); return -1; }
            if (what == WEMA_CUDA_READ_GRAY_IN) return rd(q.gray_in[channel], g.pixels, false);
            return rd(q.rec[channel][0], g.pixels, h16);
        case WEMA_CUDA_READ_ORIG6: return rd6(q.coef[channel], h16);
        case WEMA_CUDA_READ_DELTA6: return rd6(q.delta[channel], h16);
        case WEMA_CUDA_READ_AMP6:
            if (!S.materialize_amplified()) return -1;
            return rd6(S.ampl[channel], false);
        case WEMA_CUDA_READ_LOWPASS: return rd(q.ll[channel][g.levels - 1], g.low_n, false);
        case WEMA_CUDA_READ_THRESHOLD: return rd(q.thr, S.nch, false);
        case WEMA_CUDA_READ_MAGSUM: return rd(q.thr + 4, S.nch, false);
    }
    set_error("unknown stage %d", what);
    return -1;
}

WEMA_API int wema_cuda_set_timing(wema_cuda_session* s, int enable) {
    clear_error();
    if (!s) { set_error("null session"); return -1; }
    Session& S = s->s;
    if (!cuda_ok(cudaSetDevice(S.cfg.device), "cudaSetDevice")) return -1;
    if (!S.collect_timing()) return -1;
    S.timing = enable != 0;
    for (double& v : S.stage_ms) v = 0.0;
    S.stage_frames = 0;
    return 0;
}

WEMA_API int wema_cuda_stage_times(wema_cuda_session* s, double* times_ms, long long* frames) {
    clear_error();
    if (!s || !times_ms) { set_error("null argument"); return -1; }
    Session& S = s->s;
    if (!cuda_ok(cudaSetDevice(S.cfg.device), "cudaSetDevice")) return -1;
    if (!S.collect_timing()) return -1;
    for (int k = 0; k < Session::N_STAGE; k++) times_ms[k] = S.stage_ms[k];
    if (frames) *frames = S.stage_frames;
    return 0;
}

WEMA_API int wema_cuda_session_launches(wema_cuda_session* s, long long* launches) {
    clear_error();
    if (!s || !launches) { set_error("null argument"); return -1; }
    *launches = s->s.launches;
    return 0;
}

WEMA_API int wema_cuda_threshold_flat(const float* d_x, size_t n, int threshold_form, float* d_thr,
                                      float* d_sum, void* cuda_stream) {
    clear_error();
    if (!d_x || !d_thr || n == 0) { set_error("bad argument"); return -1; }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    void* scratch = nullptr;
    const size_t bytes = thr_scratch_bytes((long long)n);
    if (!cuda_ok(cudaMallocAsync(&scratch, bytes, st), "cudaMallocAsync")) return -1;
    ThrScratch ts{};
    thr_scratch_bind(ts, scratch, (long long)n);
    PyrView v{};
    v.coef = d_x;
    v.levels = 0;
    v.off6[0] = (long long)n;
    bool ok = cuda_ok(launch_threshold(&v, 1, &ts, d_thr, d_sum, threshold_form, 0, 0, st), "threshold");
    cudaFreeAsync(scratch, st);
    return ok ? 0 : -1;
}
