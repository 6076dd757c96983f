// refapi.cu - the reference's C API (dwt.h, iir_filter.h, temporal_filter.h,
// phase_amp.h, wema.h) implemented on the GPU, for C11 callers that link
// libwema_cuda in place of the reference's sources.
//
// Host-memory semantics are kept: inputs and outputs are the reference's host
// arrays and structs; each call copies in, runs the kernels, copies out and
// synchronises.  Temporal state (IIR state, window ring, the per-stream
// pipeline) stays on the device between calls.  Stateless calls use a
// per-host-thread device scratch and stream, so the reference's OpenMP callers
// may call them concurrently.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <new>
#include <unordered_map>
#include <vector>

#include "session.h"

extern "C" {
#include "dwt.h"
#include "iir_filter.h"
#include "phase_amp.h"
#include "temporal_filter.h"
#include "wema.h"
}

#define WEMA_API extern "C" __attribute__((visibility("default")))

namespace wema {
namespace {

// grow-only device scratch + stream for one host thread
struct ThreadScratch {
    char* p = nullptr;
    size_t cap = 0;
    cudaStream_t st = nullptr;
    int dev = -1;
    ~ThreadScratch() {
        if (st) cudaStreamDestroy(st);
        if (p) cudaFree(p);
    }
    bool ready() {
        int d = 0;
        if (!cuda_ok(cudaGetDevice(&d), "cudaGetDevice")) return false;
        if (!ensure_device(d)) return false;
        if (d != dev) {   // first use, or the caller switched devices
            if (st) cudaStreamDestroy(st);
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            st = nullptr;
            dev = d;
            if (!cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate"))
                return false;
        }
        return true;
    }
    char* get(size_t bytes) {
        if (!ready()) return nullptr;
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            if (!cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc(scratch)")) return nullptr;
            cap = bytes;
        }
        return p;
    }
};
thread_local ThreadScratch tls;

struct Carve {   // 256-byte aligned sub-buffers of one scratch block
    size_t off = 0;
    char* base = nullptr;
    template <class T>
    T* take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T* r = base ? (T*)(base + off) : nullptr;
        off += n * sizeof(T);
        return r;
    }
};

bool sync(cudaStream_t st) { return cuda_ok(cudaStreamSynchronize(st), "sync"); }

// 6-slot host DWTCoeffs <-> unique device planes
bool upload_slots(const DWTCoeffs* c, const Geom& g, float* d_coef, cudaStream_t st) {
    for (int l = 0; l < g.levels; l++)
        for (int b = 0; b < 3; b++)
            if (!cuda_ok(cudaMemcpyAsync(d_coef + g.uoff[l] + b * g.n[l], c->subbands[l][b].coeffs,
                                         g.n[l] * sizeof(float), cudaMemcpyHostToDevice, st),
                         "H2D"))
                return false;
    return true;
}

bool download_slots(const float* d_coef, const Geom& g, DWTCoeffs* c, cudaStream_t st) {
    for (int l = 0; l < g.levels; l++)
        for (int s = 0; s < 6; s++) {
            const int b = s < 3 ? s : 5 - s;
            if (!cuda_ok(cudaMemcpyAsync(c->subbands[l][s].coeffs, d_coef + g.uoff[l] + b * g.n[l],
                                         g.n[l] * sizeof(float), cudaMemcpyDeviceToHost, st),
                         "D2H"))
                return false;
        }
    return true;
}

bool run_forward(const Geom& g, const float* d_img, float* d_coef, float* const* d_ll,
                 cudaStream_t st) {
    for (int l = 0; l < g.levels; l++) {
        FwdLevelParams p{};
        p.iw = g.in_w[l];
        p.ih = g.in_h[l];
        p.sw = g.sw[l];
        p.sh = g.sh[l];
        p.n = g.n[l];
        p.src_planes[0] = l == 0 ? d_img : d_ll[l - 1];
        p.coef[0] = d_coef + g.uoff[l];
        p.prev[0] = l > 0 ? d_coef + g.uoff[l - 1] : nullptr;
        p.prev_n = l > 0 ? g.n[l - 1] : 0;
        p.ll_out[0] = d_ll[l];
        if (!cuda_ok(launch_dwt_fwd(kSrcPlanes, 1, p, st), "forward DWT")) return false;
    }
    return true;
}

__global__ void k_luma(const float* rgb, long long n, long long vec_end, float* y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        y[i] = i < vec_end ? luma_vec(r, g, b) : luma_tail(r, g, b);
    }
}

__global__ void k_fill(float* p, float v) { *p = v; }

IirParams flat_params(const float c[10], long long n) {
    IirParams ip{};
    memcpy(ip.c, c, 10 * sizeof(float));
    ip.levels = 1;
    ip.uoff[0] = 0;
    ip.uoff[1] = n;
    ip.off6[0] = 0;
    ip.off6[1] = n;
    ip.n[0] = n;
    ip.simd_end = n & ~15LL;
    return ip;
}

// device side of an IIRTemporalFilter, reached through filt->state_soa
struct IirImpl {
    BiquadStateSoA soa[IIR_MAX_SECTIONS];   // first member: state_soa points here
    float4* d_state = nullptr;
    float c[10];
    int dev = 0;
};
IirImpl* impl_of(const IIRTemporalFilter* f) { return reinterpret_cast<IirImpl*>(f->state_soa); }

// WemaContext -> Session
std::mutex g_ctx_mu;
std::unordered_map<const WemaContext*, Session*> g_sessions;

Session* session_of(const WemaContext* ctx) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_sessions.find(ctx);
    return it == g_sessions.end() ? nullptr : it->second;
}

Session* session_for(WemaContext* ctx) {
    Session* s = session_of(ctx);
    if (s) {
        if (s->cfg.color_mode != (int)ctx->color_mode || s->cfg.use_iir != (int)ctx->use_iir) {
            set_error("colour / temporal mode changed after the first frame");
            return nullptr;
        }
        s->cfg.edge_aware = ctx->edge_aware;
        s->cfg.bilateral_temp = ctx->bilateral_temp;
        s->cfg.amp_factor = ctx->amp_factor;
        return s;
    }
    wema_cuda_config c{};
    c.width = ctx->width;
    c.height = ctx->height;
    c.fps = ctx->fps;
    c.amp_factor = ctx->amp_factor;
    c.f_low = ctx->f_low;
    c.f_high = ctx->f_high;
    c.temporal_window = ctx->temporal_window;
    c.edge_aware = ctx->edge_aware;
    c.bilateral_temp = ctx->bilateral_temp;
    c.color_mode = ctx->color_mode;
    c.use_iir = ctx->use_iir;
    c.threshold_form = WEMA_CUDA_THR_SINGLE;
    int dev = 0;
    cudaGetDevice(&dev);
    c.device = dev;
    s = new (std::nothrow) Session();
    if (!s || !s->init(c)) {
        delete s;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    g_sessions[ctx] = s;
    return s;
}

void sync_counters(WemaContext* ctx, const Session* s) {
    if (ctx->use_iir) {
        for (IIRTemporalFilter* f : {ctx->iir_filt, ctx->iir_filt_cb, ctx->iir_filt_cr})
            if (f) f->frames_processed = s->frames_processed;
    } else {
        for (TemporalBuffer* b : {ctx->temporal_buf, ctx->temporal_buf_cb, ctx->temporal_buf_cr})
            if (b) {
                b->head = s->head;
                b->filled = s->filled;
            }
    }
}

// one frame of float RGB host data through a session
bool session_frame(Session* s, const float* in, float* out) {
    if (!s->ensure_staging()) return false;
    const size_t P3 = 3 * (size_t)s->g.pixels;
    float* d_in = s->stage_f32;
    float* d_out = s->stage_f32 + P3;
    if (!s->sync_all()) return false;   // staging reuse: the previous frame is complete
    if (!cuda_ok(cudaMemcpyAsync(d_in, in, P3 * sizeof(float), cudaMemcpyHostToDevice, s->s_fwd),
                 "H2D"))
        return false;
    if (!s->run(nullptr, d_in, nullptr, d_out, nullptr, nullptr)) return false;
    if (!cuda_ok(cudaMemcpyAsync(out, d_out, P3 * sizeof(float), cudaMemcpyDeviceToHost, s->s_inv),
                 "D2H"))
        return false;
    return sync(s->s_inv);
}

}  // namespace
}  // namespace wema

using namespace wema;

// ====================================================================== dwt.h

WEMA_API int dwt_compute_levels(int width, int height) { return compute_levels(width, height); }

WEMA_API int dwt_init(DWTCoeffs* coeffs, int width, int height, int num_levels) {
    memset(coeffs, 0, sizeof *coeffs);
    coeffs->orig_width = width;
    coeffs->orig_height = height;
    coeffs->num_levels = num_levels;
    if (num_levels < 1 || num_levels > WEMA_MAX_LEVELS || width < 1 || height < 1) return -1;
    if ((long long)width * height > (1LL << 28)) return -1;   // the kernels' 32-bit indexing
    int w = width, h = height;
    for (int l = 0; l < num_levels; l++) {
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            coeffs->subbands[l][o].width = w;
            coeffs->subbands[l][o].height = h;
            coeffs->subbands[l][o].coeffs = (float*)calloc((size_t)w * h, sizeof(float));
            if (!coeffs->subbands[l][o].coeffs) {
                dwt_free(coeffs);
                return -1;
            }
        }
    }
    coeffs->lowpass_w = w;
    coeffs->lowpass_h = h;
    coeffs->lowpass = (float*)calloc((size_t)w * h, sizeof(float));
    if (!coeffs->lowpass) {
        dwt_free(coeffs);
        return -1;
    }
    return 0;
}

WEMA_API void dwt_free(DWTCoeffs* coeffs) {
    for (int l = 0; l < WEMA_MAX_LEVELS; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            free(coeffs->subbands[l][o].coeffs);
            coeffs->subbands[l][o].coeffs = nullptr;
        }
    free(coeffs->lowpass);
    coeffs->lowpass = nullptr;
}

WEMA_API size_t dwt_num_positions(const DWTCoeffs* coeffs) {
    size_t t = 0;
    for (int l = 0; l < coeffs->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++)
            t += (size_t)coeffs->subbands[l][o].width * coeffs->subbands[l][o].height;
    return t;
}

WEMA_API void dwt_forward(const float* image, int width, int height, DWTCoeffs* coeffs) {
    clear_error();
    const Geom g = make_geom(width, height, coeffs->num_levels);
    Carve c;
    c.take<float>(g.pixels);
    c.take<float>(g.uoff[g.levels]);
    for (int l = 0; l < g.levels; l++) c.take<float>(g.n[l]);
    char* base = tls.get(c.off);
    if (!base) return;
    c = Carve();
    c.base = base;
    float* d_img = c.take<float>(g.pixels);
    float* d_coef = c.take<float>(g.uoff[g.levels]);
    float* d_ll[WEMA_MAX_LEV];
    for (int l = 0; l < g.levels; l++) d_ll[l] = c.take<float>(g.n[l]);
    cudaStream_t st = tls.st;
    if (!cuda_ok(cudaMemcpyAsync(d_img, image, g.pixels * sizeof(float), cudaMemcpyHostToDevice, st),
                 "H2D"))
        return;
    if (!run_forward(g, d_img, d_coef, d_ll, st)) return;
    if (!download_slots(d_coef, g, coeffs, st)) return;
    cuda_ok(cudaMemcpyAsync(coeffs->lowpass, d_ll[g.levels - 1], g.low_n * sizeof(float),
                            cudaMemcpyDeviceToHost, st),
            "D2H");
    sync(st);
}

WEMA_API void dwt_inverse(const DWTCoeffs* coeffs, float* image) {
    clear_error();
    const Geom g = make_geom(coeffs->orig_width, coeffs->orig_height, coeffs->num_levels);
    Carve c;
    c.take<float>(g.uoff[g.levels]);
    c.take<float>(g.low_n);
    for (int l = 0; l < g.levels; l++) c.take<float>((size_t)g.in_w[l] * g.in_h[l]);
    c.take<float>(4);
    char* base = tls.get(c.off);
    if (!base) return;
    c = Carve();
    c.base = base;
    float* d_coef = c.take<float>(g.uoff[g.levels]);
    float* d_low = c.take<float>(g.low_n);
    float* d_rec[WEMA_MAX_LEV];
    for (int l = 0; l < g.levels; l++) d_rec[l] = c.take<float>((size_t)g.in_w[l] * g.in_h[l]);
    float* d_inf = c.take<float>(4);
    cudaStream_t st = tls.st;
    if (!upload_slots(coeffs, g, d_coef, st)) return;
    if (!cuda_ok(cudaMemcpyAsync(d_low, coeffs->lowpass, g.low_n * sizeof(float),
                                 cudaMemcpyHostToDevice, st),
                 "H2D"))
        return;
    k_fill<<<1, 1, 0, st>>>(d_inf, INFINITY);   // no coefficient passes an infinite threshold
    for (int l = g.levels - 1; l >= 0; l--) {
        InvLevelParams q{};
        q.ow = g.in_w[l];
        q.oh = g.in_h[l];
        q.sw = g.sw[l];
        q.sh = g.sh[l];
        q.n = g.n[l];
        q.ll[0] = l == g.levels - 1 ? d_low : d_rec[l + 1];
        q.coef[0] = d_coef + g.uoff[l];
        q.delta[0] = d_coef + g.uoff[l];
        q.thr = d_inf;
        q.out_planes[0] = d_rec[l];
        if (!cuda_ok(launch_dwt_inv(1, kOutPlanes, q, st), "inverse DWT")) return;
    }
    if (!cuda_ok(cudaMemcpyAsync(image, d_rec[0], g.pixels * sizeof(float), cudaMemcpyDeviceToHost, st),
                 "D2H"))
        return;
    sync(st);
}

// =============================================================== iir_filter.h

WEMA_API int iir_design_bandpass(IIRFilterCoeffs* coeffs, float f_low, float f_high, float fs,
                                 int order) {
    memset(coeffs, 0, sizeof *coeffs);
    float c[10];
    if (design_bandpass(f_low, f_high, fs, c, nullptr) < 0) return -1;
    if (order < 2) order = 2;
    if (order > 4) order = 4;
    const int per = order / 2;
    coeffs->num_sections = 2 * per;
    for (int i = 0; i < per; i++) {
        coeffs->sections[i] = BiquadCoeffs{c[0], c[1], c[2], c[3], c[4]};
        coeffs->sections[per + i] = BiquadCoeffs{c[5], c[6], c[7], c[8], c[9]};
    }
    return 0;
}

WEMA_API int iir_temporal_init(IIRTemporalFilter* filt, size_t num_positions, float f_low,
                               float f_high, float fs) {
    clear_error();
    memset(filt, 0, sizeof *filt);
    if (iir_design_bandpass(&filt->coeffs, f_low, f_high, fs, 2) < 0) return -1;
    filt->num_positions = num_positions;
    IirImpl* im = new (std::nothrow) IirImpl();
    if (!im) return -1;
    if (design_bandpass(f_low, f_high, fs, im->c, &filt->warmup_frames) < 0) {
        delete im;
        return -1;
    }
    if (!tls.ready() || !cuda_ok(cudaGetDevice(&im->dev), "cudaGetDevice") ||
        !cuda_ok(cudaMalloc(&im->d_state, num_positions * sizeof(float4) + 16), "cudaMalloc(state)") ||
        !cuda_ok(cudaMemset(im->d_state, 0, num_positions * sizeof(float4) + 16), "cudaMemset")) {
        if (im->d_state) cudaFree(im->d_state);
        delete im;
        return -1;
    }
    for (int s = 0; s < 2; s++) {   // device pointers; the layout is one float4 per position
        im->soa[s].w1 = reinterpret_cast<float*>(im->d_state) + 2 * s;
        im->soa[s].w2 = reinterpret_cast<float*>(im->d_state) + 2 * s + 1;
    }
    filt->state = nullptr;
    filt->state_soa = im->soa;
    filt->use_simd = true;
    filt->frames_processed = 0;
    return 0;
}

WEMA_API void iir_temporal_free(IIRTemporalFilter* filt) {
    if (filt->state_soa) {
        IirImpl* im = impl_of(filt);
        cudaFree(im->d_state);
        delete im;
        filt->state_soa = nullptr;
    }
    filt->state = nullptr;
    filt->num_positions = 0;
}

static bool iir_frames(IIRTemporalFilter* filt, const float* in, float* out, int frames,
                       bool preseed) {
    clear_error();
    IirImpl* im = impl_of(filt);
    if (!im) { set_error("filter not initialised"); return false; }
    const long long n = (long long)filt->num_positions;
    const size_t bytes = (size_t)n * frames * sizeof(float);
    char* base = tls.get(2 * bytes + 512);
    if (!base) return false;
    float* d_in = (float*)base;
    float* d_out = (float*)(base + ((bytes + 255) & ~(size_t)255));
    cudaStream_t st = tls.st;
    if (!cuda_ok(cudaMemcpyAsync(d_in, in, bytes, cudaMemcpyHostToDevice, st), "H2D")) return false;
    const IirParams ip = flat_params(im->c, n);
    if (preseed) {
        if (!cuda_ok(launch_iir_preseed(ip, d_in, im->d_state, 0, filt->warmup_frames, st), "preseed"))
            return false;
        return sync(st);
    }
    for (int f = 0; f < frames; f++)
        if (!cuda_ok(launch_iir(ip, d_in + f * n, im->d_state, 0, d_out + f * n, st), "IIR")) return false;
    if (!cuda_ok(cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st), "D2H")) return false;
    return sync(st);
}

WEMA_API void iir_temporal_process(IIRTemporalFilter* filt, const float* input, float* output) {
    if (iir_frames(filt, input, output, 1, false)) filt->frames_processed++;
}

WEMA_API void iir_temporal_process_batch(IIRTemporalFilter* filt, const float* input,
                                         float* output, int batch_size) {
    if (batch_size <= 0) return;
    if (iir_frames(filt, input, output, batch_size, false)) filt->frames_processed += batch_size;
}

WEMA_API bool iir_temporal_ready(const IIRTemporalFilter* filt) {
    return filt->frames_processed >= filt->warmup_frames;
}

WEMA_API void iir_temporal_preseed(IIRTemporalFilter* filt, const float* initial_coeffs) {
    if (filt->frames_processed > 0) return;
    if (iir_frames(filt, initial_coeffs, nullptr, 1, true))
        filt->frames_processed = filt->warmup_frames;
}

// ========================================================= temporal_filter.h

WEMA_API int temporal_filter_init(TemporalFilter* filt, float f_low, float f_high, int window_size) {
    memset(filt, 0, sizeof *filt);
    filt->f_low_norm = f_low;
    filt->f_high_norm = f_high;
    int levels = 0;
    for (int ws = window_size; ws > 1; ws /= 2) levels++;
    filt->temporal_levels = levels;
    filt->filter_len = 2;
    filt->lp_filter = (float*)malloc(2 * sizeof(float));
    filt->hp_filter = (float*)malloc(2 * sizeof(float));
    if (!filt->lp_filter || !filt->hp_filter) {
        temporal_filter_free(filt);
        return -1;
    }
    filt->lp_filter[0] = filt->lp_filter[1] = 0.5f;   // Haar pair (temporal_filter.c:82-85)
    filt->hp_filter[0] = 0.5f;
    filt->hp_filter[1] = -0.5f;
    return 0;
}

WEMA_API void temporal_filter_free(TemporalFilter* filt) {
    free(filt->lp_filter);
    free(filt->hp_filter);
    filt->lp_filter = nullptr;
    filt->hp_filter = nullptr;
}

WEMA_API int temporal_buffer_init(TemporalBuffer* buf, const DWTCoeffs* coeffs, int window_size) {
    clear_error();
    memset(buf, 0, sizeof *buf);
    buf->window_size = window_size;
    buf->num_levels = coeffs->num_levels;
    size_t total = 0;
    for (int l = 0; l < coeffs->num_levels; l++) {
        buf->widths[l] = coeffs->subbands[l][0].width;
        buf->heights[l] = coeffs->subbands[l][0].height;
        total += (size_t)buf->widths[l] * buf->heights[l] * WEMA_NUM_ORIENTATIONS;
    }
    buf->num_positions = total;
    if (window_size < 1 || window_size > WEMA_TEMPORAL_WINDOW_MAX) {
        set_error("window size must be in 1..%d", WEMA_TEMPORAL_WINDOW_MAX);
        return -1;
    }
    buf->amplitude = (float*)calloc(total, sizeof(float));
    buf->dc_phase = (float*)calloc(total, sizeof(float));
    if (!buf->amplitude || !buf->dc_phase || !tls.ready() ||
        !cuda_ok(cudaMalloc(&buf->phase_buffer, total * window_size * sizeof(float)), "cudaMalloc(ring)") ||
        !cuda_ok(cudaMemset(buf->phase_buffer, 0, total * window_size * sizeof(float)), "cudaMemset")) {
        temporal_buffer_free(buf);
        return -1;
    }
    return 0;
}

WEMA_API void temporal_buffer_free(TemporalBuffer* buf) {
    if (buf->phase_buffer) cudaFree(buf->phase_buffer);
    free(buf->amplitude);
    free(buf->dc_phase);
    buf->phase_buffer = nullptr;
    buf->amplitude = nullptr;
    buf->dc_phase = nullptr;
}

WEMA_API void temporal_buffer_push(TemporalBuffer* buf, const DWTCoeffs* coeffs) {
    clear_error();
    size_t pos = 0;
    for (int l = 0; l < coeffs->num_levels; l++)
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++) {
            const size_t n = (size_t)coeffs->subbands[l][o].width * coeffs->subbands[l][o].height;
            memcpy(buf->amplitude + pos, coeffs->subbands[l][o].coeffs, n * sizeof(float));
            pos += n;
        }
    if (!tls.ready()) return;
    if (!cuda_ok(cudaMemcpyAsync(buf->phase_buffer + (size_t)buf->head * buf->num_positions,
                                 buf->amplitude, buf->num_positions * sizeof(float),
                                 cudaMemcpyHostToDevice, tls.st),
                 "H2D") ||
        !sync(tls.st))
        return;
    buf->head = (buf->head + 1) % buf->window_size;
    if (buf->filled < buf->window_size) buf->filled++;
}

WEMA_API void temporal_filter_apply(const TemporalFilter* filt, const TemporalBuffer* buf,
                                    float* delta_phi_filtered, bool bilateral) {
    (void)filt;
    clear_error();
    if (buf->filled < buf->window_size) {
        memset(delta_phi_filtered, 0, buf->num_positions * sizeof(float));
        return;
    }
    float* d_delta = (float*)tls.get(buf->num_positions * sizeof(float));
    if (!d_delta) return;
    WindowParams wp{};
    wp.pu = (long long)buf->num_positions;
    wp.ws = buf->window_size;
    wp.head = buf->head;
    wp.bilateral = bilateral;
    const int ws = buf->window_size, center = ws / 2;
    const float ts = (float)ws * 0.15f;
    const float inv2 = 0.5f / (ts * ts);
    for (int t = 0; t < ws; t++) {
        const float d = (float)(t - center);
        wp.time_w[t] = expf(-(d * d) * inv2);
    }
    if (!cuda_ok(launch_window(wp, buf->phase_buffer, d_delta, tls.st), "window filter")) return;
    if (!cuda_ok(cudaMemcpyAsync(delta_phi_filtered, d_delta, buf->num_positions * sizeof(float),
                                 cudaMemcpyDeviceToHost, tls.st),
                 "D2H"))
        return;
    sync(tls.st);
}

WEMA_API int temporal_buffer_output_count(const TemporalBuffer* buf) {
    if (buf->filled < buf->window_size) return 0;
    return buf->filled - buf->window_size / 2;
}

// =============================================================== phase_amp.h

WEMA_API void coeff_amplify(const float* delta_coeff, const float* orig_coeff, float alpha,
                            DWTCoeffs* coeffs) {
    clear_error();
    // total over the six slots from slot 0's dims (phase_amp.c:17-22)
    long long off[WEMA_MAX_LEVELS + 1];
    long long total = 0;
    for (int l = 0; l < coeffs->num_levels; l++) {
        off[l] = total;
        total += 6LL * coeffs->subbands[l][0].width * coeffs->subbands[l][0].height;
    }
    off[coeffs->num_levels] = total;
    if (total == 0) return;
    const size_t bytes = (size_t)total * sizeof(float);
    const size_t sb = thr_scratch_bytes(total);
    Carve c;
    c.take<float>(total);
    c.take<float>(total);
    c.take<float>(total);
    c.take<float>(8);
    c.take<char>(sb);
    char* base = tls.get(c.off);
    if (!base) return;
    c = Carve();
    c.base = base;
    float* d_orig = c.take<float>(total);
    float* d_delta = c.take<float>(total);
    float* d_out = c.take<float>(total);
    float* d_thr = c.take<float>(8);
    void* scratch = c.take<char>(sb);
    cudaStream_t st = tls.st;
    if (!cuda_ok(cudaMemcpyAsync(d_orig, orig_coeff, bytes, cudaMemcpyHostToDevice, st), "H2D") ||
        !cuda_ok(cudaMemcpyAsync(d_delta, delta_coeff, bytes, cudaMemcpyHostToDevice, st), "H2D"))
        return;
    ThrScratch ts{};
    thr_scratch_bind(ts, scratch, total);
    PyrView v{};
    v.coef = d_orig;
    v.levels = 0;
    v.off6[0] = total;
    if (!cuda_ok(launch_threshold(&v, 1, &ts, d_thr, nullptr, WEMA_CUDA_THR_SINGLE, 0, 0, st), "threshold"))
        return;
    IirParams ip{};
    ip.levels = coeffs->num_levels;
    for (int l = 0; l <= coeffs->num_levels; l++) ip.uoff[l] = ip.off6[l] = off[l];
    if (!cuda_ok(launch_amplify(ip, d_orig, d_delta, d_thr, alpha, d_out, st), "amplify")) return;
    for (int l = 0; l < coeffs->num_levels; l++) {
        const long long n = (long long)coeffs->subbands[l][0].width * coeffs->subbands[l][0].height;
        for (int o = 0; o < WEMA_NUM_ORIENTATIONS; o++)
            if (!cuda_ok(cudaMemcpyAsync(coeffs->subbands[l][o].coeffs, d_out + off[l] + o * n,
                                         n * sizeof(float), cudaMemcpyDeviceToHost, st),
                         "D2H"))
                return;
    }
    sync(st);
}

// ==================================================================== wema.h

WEMA_API int frame_alloc(Frame* frame, int width, int height, int channels) {
    frame->width = width;
    frame->height = height;
    frame->channels = channels;
    frame->data = (float*)calloc((size_t)width * height * channels, sizeof(float));
    return frame->data ? 0 : -1;
}

WEMA_API void frame_free(Frame* frame) {
    free(frame->data);
    frame->data = nullptr;
}

WEMA_API void frame_rgb_to_gray(const Frame* rgb, float* gray) {
    clear_error();
    const long long n = (long long)rgb->width * rgb->height;
    char* base = tls.get((size_t)n * 16 + 256);
    if (!base) return;
    float* d_rgb = (float*)base;
    float* d_y = d_rgb + 3 * n + 64;
    cudaStream_t st = tls.st;
    if (!cuda_ok(cudaMemcpyAsync(d_rgb, rgb->data, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D"))
        return;
    k_luma<<<(int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, st>>>(d_rgb, n, vec_cover(n), d_y);
    if (!cuda_ok(cudaGetLastError(), "luma") ||
        !cuda_ok(cudaMemcpyAsync(gray, d_y, n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H"))
        return;
    sync(st);
}

// Gaussian-fallback transfer (wema.c:338-353).  delta_buf and smooth_buf are
// the reference's scratch; they are not filled here.
WEMA_API void frame_gray_to_rgb(const float* gray, const Frame* orig, Frame* out,
                                float* delta_buf, float* smooth_buf) {
    (void)delta_buf;
    (void)smooth_buf;
    clear_error();
    const long long n = (long long)orig->width * orig->height;
    char* base = tls.get((size_t)n * 28 + 512);
    if (!base) return;
    float* d_rgb = (float*)base;
    float* d_gray = d_rgb + 3 * n + 64;
    float* d_out = d_gray + n + 64;
    cudaStream_t st = tls.st;
    if (!cuda_ok(cudaMemcpyAsync(d_rgb, orig->data, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D") ||
        !cuda_ok(cudaMemcpyAsync(d_gray, gray, n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D"))
        return;
    TransferParams tp{};
    tp.w = orig->width;
    tp.h = orig->height;
    tp.vec_end = vec_cover(n);
    tp.src_f32 = d_rgb;
    tp.gray_out = d_gray;
    tp.out_f32 = d_out;
    tp.edge_aware = 0;
    if (!cuda_ok(launch_transfer(tp, st), "transfer") ||
        !cuda_ok(cudaMemcpyAsync(out->data, d_out, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H"))
        return;
    sync(st);
}

WEMA_API int wema_init(WemaContext* ctx, int width, int height, float fps, float amp_factor,
                       float f_low, float f_high, int temporal_window) {
    clear_error();
    memset(ctx, 0, sizeof *ctx);
    ctx->width = width;
    ctx->height = height;
    ctx->fps = fps;
    ctx->amp_factor = amp_factor;
    ctx->f_low = f_low;
    ctx->f_high = f_high;
    ctx->temporal_window = temporal_window;
    ctx->edge_aware = true;       // wema.c:371-373
    ctx->bilateral_temp = true;
    ctx->color_mode = false;
    ctx->f_low_norm = f_low / (fps / 2.0f);
    ctx->f_high_norm = f_high / (fps / 2.0f);
    if (ctx->f_low_norm < 0.0f) ctx->f_low_norm = 0.0f;
    if (ctx->f_high_norm > 1.0f) ctx->f_high_norm = 1.0f;
    ctx->num_levels = dwt_compute_levels(width, height);
    ctx->coeffs = (DWTCoeffs*)calloc(1, sizeof(DWTCoeffs));
    ctx->temporal_buf = (TemporalBuffer*)calloc(1, sizeof(TemporalBuffer));
    ctx->temporal_filt = (TemporalFilter*)calloc(1, sizeof(TemporalFilter));
    if (!ctx->coeffs || !ctx->temporal_buf || !ctx->temporal_filt ||
        dwt_init(ctx->coeffs, width, height, ctx->num_levels) < 0 ||
        temporal_filter_init(ctx->temporal_filt, ctx->f_low_norm, ctx->f_high_norm, temporal_window) < 0) {
        wema_free(ctx);
        return -1;
    }
    // window-mode counters; the ring itself lives in the stream's device session
    ctx->temporal_buf->window_size = temporal_window;
    ctx->temporal_buf->num_levels = ctx->num_levels;
    ctx->temporal_buf->num_positions = dwt_num_positions(ctx->coeffs);
    for (int l = 0; l < ctx->num_levels; l++) {
        ctx->temporal_buf->widths[l] = ctx->coeffs->subbands[l][0].width;
        ctx->temporal_buf->heights[l] = ctx->coeffs->subbands[l][0].height;
    }
    return 0;
}

WEMA_API int wema_init_color(WemaContext* ctx) {
    ctx->coeffs_cb = (DWTCoeffs*)calloc(1, sizeof(DWTCoeffs));
    ctx->coeffs_cr = (DWTCoeffs*)calloc(1, sizeof(DWTCoeffs));
    ctx->temporal_buf_cb = (TemporalBuffer*)calloc(1, sizeof(TemporalBuffer));
    ctx->temporal_buf_cr = (TemporalBuffer*)calloc(1, sizeof(TemporalBuffer));
    if (!ctx->coeffs_cb || !ctx->coeffs_cr || !ctx->temporal_buf_cb || !ctx->temporal_buf_cr)
        return -1;
    if (dwt_init(ctx->coeffs_cb, ctx->width, ctx->height, ctx->num_levels) < 0 ||
        dwt_init(ctx->coeffs_cr, ctx->width, ctx->height, ctx->num_levels) < 0)
        return -1;
    for (TemporalBuffer* b : {ctx->temporal_buf_cb, ctx->temporal_buf_cr}) {
        b->window_size = ctx->temporal_window;
        b->num_levels = ctx->num_levels;
        b->num_positions = dwt_num_positions(ctx->coeffs_cb);
    }
    return 0;
}

static IIRTemporalFilter* host_iir(const WemaContext* ctx) {
    IIRTemporalFilter* f = (IIRTemporalFilter*)calloc(1, sizeof(IIRTemporalFilter));
    if (!f) return nullptr;
    float c[10];
    if (iir_design_bandpass(&f->coeffs, ctx->f_low, ctx->f_high, ctx->fps, 2) < 0 ||
        design_bandpass(ctx->f_low, ctx->f_high, ctx->fps, c, &f->warmup_frames) < 0) {
        free(f);
        return nullptr;
    }
    f->num_positions = dwt_num_positions(ctx->coeffs);
    f->use_simd = true;   // state lives in the stream's device session
    return f;
}

WEMA_API int wema_init_iir(WemaContext* ctx) {
    clear_error();
    ctx->iir_filt = host_iir(ctx);
    if (!ctx->iir_filt) {
        set_error("invalid band: need 0 < f_low < f_high < fps/2");
        return -1;
    }
    if (ctx->temporal_buf) {   // wema.c:508-518: the window state is not needed
        free(ctx->temporal_buf);
        ctx->temporal_buf = nullptr;
    }
    if (ctx->temporal_filt) {
        temporal_filter_free(ctx->temporal_filt);
        free(ctx->temporal_filt);
        ctx->temporal_filt = nullptr;
    }
    ctx->use_iir = true;
    return 0;
}

WEMA_API int wema_init_iir_color(WemaContext* ctx) {
    if (!ctx->coeffs_cb || !ctx->coeffs_cr) return -1;
    ctx->iir_filt_cb = host_iir(ctx);
    ctx->iir_filt_cr = host_iir(ctx);
    if (!ctx->iir_filt_cb || !ctx->iir_filt_cr) return -1;
    free(ctx->temporal_buf_cb);
    free(ctx->temporal_buf_cr);
    ctx->temporal_buf_cb = ctx->temporal_buf_cr = nullptr;
    return 0;
}

WEMA_API void wema_free(WemaContext* ctx) {
    {
        std::lock_guard<std::mutex> lk(g_ctx_mu);
        auto it = g_sessions.find(ctx);
        if (it != g_sessions.end()) {
            cudaSetDevice(it->second->cfg.device);
            delete it->second;
            g_sessions.erase(it);
        }
    }
    for (DWTCoeffs** c : {&ctx->coeffs, &ctx->coeffs_cb, &ctx->coeffs_cr})
        if (*c) {
            dwt_free(*c);
            free(*c);
            *c = nullptr;
        }
    for (TemporalBuffer** b : {&ctx->temporal_buf, &ctx->temporal_buf_cb, &ctx->temporal_buf_cr})
        if (*b) {
            free(*b);
            *b = nullptr;
        }
    if (ctx->temporal_filt) {
        temporal_filter_free(ctx->temporal_filt);
        free(ctx->temporal_filt);
        ctx->temporal_filt = nullptr;
    }
    for (IIRTemporalFilter** f : {&ctx->iir_filt, &ctx->iir_filt_cb, &ctx->iir_filt_cr}) {
        free(*f);
        *f = nullptr;
    }
}

WEMA_API bool wema_ready(const WemaContext* ctx) {
    if (ctx->use_iir) return ctx->iir_filt && iir_temporal_ready(ctx->iir_filt);
    return ctx->temporal_buf && temporal_buffer_ready(ctx->temporal_buf);
}

WEMA_API int wema_process_frame(WemaContext* ctx, const Frame* in, Frame* out) {
    clear_error();
    if (!in || !out || !in->data || !out->data || in->width != ctx->width ||
        in->height != ctx->height || in->channels != 3) {
        set_error("frames must be %dx%d RGB with data", ctx->width, ctx->height);
        return -1;
    }
    Session* s = session_for(ctx);
    if (!s) return -1;
    s->cfg.threshold_form = WEMA_CUDA_THR_SINGLE;
    if (!session_frame(s, in->data, out->data)) return -1;
    sync_counters(ctx, s);
    return 0;
}

WEMA_API int wema_flush(WemaContext* ctx, Frame* out) {
    (void)ctx;
    (void)out;
    return -1;   // wema.c:954-960
}

WEMA_API int wema_batch_init(WemaBatchContext* batch, const WemaContext* wema, int batch_size,
                             int num_threads) {
    memset(batch, 0, sizeof *batch);
    if (batch_size < 1) batch_size = WEMA_BATCH_SIZE_DEF;
    if (batch_size > WEMA_BATCH_SIZE_MAX) batch_size = WEMA_BATCH_SIZE_MAX;
    batch->batch_size = batch_size;
    batch->width = wema->width;
    batch->height = wema->height;
    batch->num_threads = num_threads > 0 ? num_threads : 1;
    batch->num_positions = wema->coeffs ? dwt_num_positions(wema->coeffs) : 0;
    batch->smooth_buf_stride = 9 * wema->width * wema->height;
    return 0;
}

WEMA_API void wema_batch_free(WemaBatchContext* batch) { memset(batch, 0, sizeof *batch); }

// The batch route (wema_batch.c:352-457): IIR luma with the guided filter
// always on and the threshold in its (0.2/N)*sum form; frames run in order on
// the stream's device state.
WEMA_API int wema_batch_process(WemaContext* wema, WemaBatchContext* batch, const Frame* frames_in,
                                Frame* frames_out, int frame_count) {
    clear_error();
    if (frame_count <= 0) return 0;
    if (frame_count > batch->batch_size) frame_count = batch->batch_size;
    if (!wema->use_iir || wema->color_mode) {
        set_error("the batch route processes IIR luma only");
        return -1;
    }
    Session* s = session_for(wema);
    if (!s) return -1;
    const int edge = s->cfg.edge_aware;
    s->cfg.threshold_form = WEMA_CUDA_THR_BATCH;
    s->cfg.edge_aware = 1;
    int done = 0;
    for (; done < frame_count; done++)
        if (!session_frame(s, frames_in[done].data, frames_out[done].data)) break;
    s->cfg.edge_aware = edge;
    s->cfg.threshold_form = WEMA_CUDA_THR_SINGLE;
    sync_counters(wema, s);
    return done == frame_count ? frame_count : -1;
}
