/*
 * wema_cuda.h - extensions of libwema_cuda beyond the reference's C API.
 *
 * The reference API (dwt.h, iir_filter.h, temporal_filter.h, phase_amp.h,
 * wema.h) keeps host-memory semantics so existing C11 callers drop in
 * unchanged.  These entry points expose what the GPU adds: sessions whose
 * state stays resident in device memory, u8 RGB24 frames on the device (no
 * float frames over PCIe), explicit CUDA streams, inspection of the
 * per-frame stages, and the HBM footprint used for admission control.
 *
 * All functions return 0 on success and -1 on error (the reference's
 * convention, wema.c:437-439); wema_cuda_last_error() then describes the
 * failure.  A session is not thread-safe: one host thread drives it.
 */
#ifndef WEMA_CUDA_H
#define WEMA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WEMA_CUDA_ABI_VERSION 2

typedef struct wema_cuda_session wema_cuda_session;

/* Threshold evaluation order: the reference's single-frame route computes
 * (sum/N)*0.2 (wema.c:723), its batch route (0.2/N)*sum (wema_batch.c:276).
 * They differ in the last bit and so can flip a mask. */
enum { WEMA_CUDA_THR_SINGLE = 0, WEMA_CUDA_THR_BATCH = 1 };

typedef struct {
    int   width, height;
    float fps;
    float amp_factor;        /* alpha (wema.h WemaContext.amp_factor) */
    float f_low, f_high;     /* Hz; IIR band, as wema_init */
    int   temporal_window;   /* window mode: ws (4..256) */
    int   edge_aware;        /* guided filter (1) or 5-tap Gaussian (0), luma only */
    int   bilateral_temp;    /* window mode: bilateral weighting */
    int   color_mode;        /* YCbCr, three pyramids, no luma transfer */
    int   use_iir;           /* 1: IIR band-pass (default), 0: window ("--haar") mode */
    int   threshold_form;    /* WEMA_CUDA_THR_SINGLE or WEMA_CUDA_THR_BATCH */
    int   device;            /* CUDA device ordinal */
    int   iir_state_fp64;    /* precision variant: biquad state and its update in FP64
                                (the FP32-designed coefficients promoted; 32 B of state
                                per position instead of 16).  0: the reference's FP32 */
    int   ring_fp16;         /* precision variant, window mode: the temporal ring stored
                                in FP16 (round to nearest), arithmetic in FP32; halves
                                the ring's bytes (read ws times per position per frame) */
    int   planes_fp16;       /* precision variant: the detail-coefficient and band-passed
                                delta planes and the reconstructed frame (the level-0
                                reconstruction) stored in FP16 (round to nearest),
                                arithmetic in FP32; the IIR state and the LL / coarser
                                reconstruction planes stay FP32.  The threshold is then the FP64 sum of the
                                FP16 coefficients rounded once, not the reference's
                                bit-exact FP32 sum: outputs are NOT within the bit-exact /
                                1-LSB parity bars of the FP32 path (their error against an
                                FP64 re-evaluation is reported instead).  0: FP32 */
} wema_cuda_config;

/* Fills *cfg with the reference CLI's defaults for a stream of the given
 * size and rate (main.c:66-75: amp 120, 0.5 Hz .. Nyquist-1e-4, window 32,
 * edge-aware on, bilateral off, IIR, luma). */
void wema_cuda_config_default(wema_cuda_config *cfg, int width, int height, float fps);

int  wema_cuda_session_create(const wema_cuda_config *cfg, wema_cuda_session **out);
void wema_cuda_session_destroy(wema_cuda_session *s);

/* Device bytes a session of this configuration holds (pyramid, IIR state or
 * window ring, threshold scratch, staging): the admission footprint. */
size_t wema_cuda_session_bytes(const wema_cuda_config *cfg);

/* One frame, device pointers.  in/out are RGB24 [height][width][3]; out may
 * not alias in.  With a `cuda_stream` (a cudaStream_t) the frame is ordered
 * after the work already queued on it and the stream waits for the output.
 * With NULL the frame is queued behind the session's earlier frames only;
 * wema_cuda_session_sync() waits for it.  Either way consecutive frames
 * overlap inside the session: frame t+1's forward transform and temporal
 * filter run while frame t's threshold and inverse finish. */
int wema_cuda_process_u8(wema_cuda_session *s, const uint8_t *d_in, uint8_t *d_out,
                         void *cuda_stream);
/* The same with explicit events (cudaEvent_t, either may be NULL): the
 * session waits for `wait_event` before reading d_in or writing d_out, and
 * records `done_event` once d_out is complete and d_in no longer read. */
int wema_cuda_process_u8_async(wema_cuda_session *s, const uint8_t *d_in, uint8_t *d_out,
                               void *wait_event, void *done_event);
/* Same with float RGB in [0,1] (the reference's Frame layout); either output
 * pointer may be NULL. */
int wema_cuda_process_f32(wema_cuda_session *s, const float *d_in, float *d_out_f32,
                          uint8_t *d_out_u8, void *cuda_stream);
/* Host RGB24 in/out; copies in, processes, copies out, synchronises. */
int wema_cuda_process_host_u8(wema_cuda_session *s, const uint8_t *h_in, uint8_t *h_out);

/* Waits for the session's queued work. */
int wema_cuda_session_sync(wema_cuda_session *s);

/* Snapshot / restore of a stream's whole state (no counterpart in the
 * reference; for moving a stream between processes or devices and for
 * recovery): the frame counters and every device buffer (IIR state or window
 * ring, threshold history, pyramids) copied to caller-owned host memory of
 * wema_cuda_session_snapshot_bytes() bytes.  Restore into a session of the same
 * configuration (any device): its next frame continues the stream exactly as
 * the original would have.  Both wait for the session's work. */
size_t wema_cuda_session_snapshot_bytes(wema_cuda_session *s);
int wema_cuda_session_snapshot(wema_cuda_session *s, void *host, size_t cap);
int wema_cuda_session_restore(wema_cuda_session *s, const void *host, size_t bytes);

/* Keep each frame's converted input planes and (colour) reconstructed planes
 * so WEMA_CUDA_READ_GRAY_IN / _GRAY_OUT can return them (off by default: they
 * cost two extra plane writes per channel and frame). */
int wema_cuda_set_inspect(wema_cuda_session *s, int enable);

/* Frames seen by the temporal filter (the reference's frames_processed,
 * which jumps to the warm-up count at the first frame's preseed). */
int wema_cuda_session_frames_processed(const wema_cuda_session *s);

/* Copies a stage of the last queued frame to host memory, in the
 * reference's layouts (waits for the session first).  Returns the element count, or
 * -1.  `what`: */
enum {
    WEMA_CUDA_READ_GRAY_IN = 0,   /* Y plane [P] (colour: Y) */
    WEMA_CUDA_READ_GRAY_OUT = 1,  /* reconstructed Y [P] */
    WEMA_CUDA_READ_ORIG6 = 2,     /* original coefficients, 6-slot flat [N6] */
    WEMA_CUDA_READ_DELTA6 = 3,    /* band-passed deltas, 6-slot [N6] (slots 3-5 mirrored) */
    WEMA_CUDA_READ_AMP6 = 4,      /* amplified coefficients, 6-slot [N6] */
    WEMA_CUDA_READ_LOWPASS = 5,   /* coarsest LL */
    WEMA_CUDA_READ_THRESHOLD = 6, /* per-channel thresholds [channels] */
    WEMA_CUDA_READ_MAGSUM = 7     /* per-channel sum |x| [channels] */
};
long wema_cuda_session_read(wema_cuda_session *s, int what, int channel, float *h_dst, size_t cap);

/* Per-stage device timing with CUDA events on each stage's stream: stages are
 * forward DWT level 0, forward DWT levels >= 1, threshold, temporal filter,
 * inverse DWT levels >= 1, inverse DWT level 0 (with the colour output),
 * luma transfer.  times_ms[7] receives the accumulated milliseconds, *frames
 * the frames timed.  No counterpart in the reference (instrumentation). */
enum { WEMA_CUDA_STAGES = 7 };
int wema_cuda_set_timing(wema_cuda_session *s, int enable);
int wema_cuda_stage_times(wema_cuda_session *s, double *times_ms, long long *frames);

/* Kernel launches this session has issued so far (all frames).  No
 * counterpart in the reference (instrumentation). */
int wema_cuda_session_launches(wema_cuda_session *s, long long *launches);

/* Exact reference threshold of a device array of n floats (plain flat
 * order), written to *d_thr; d_sum optional.  Allocates its scratch. */
int wema_cuda_threshold_flat(const float *d_x, size_t n, int threshold_form, float *d_thr,
                             float *d_sum, void *cuda_stream);

/* The same exact threshold with no device allocation (no counterpart in the
 * reference: it exists for callers that must not allocate device memory,
 * e.g. a host that owns the GPU's memory through its own pool or a real-time
 * loop that cannot absorb cudaMalloc's synchronisation).  Its scratch is a
 * fixed 4 MiB array compiled into the library, held by every device that
 * loads it; n is limited to 2^24 elements (more than a 3840x2160 frame's
 * 6-slot coefficients) and larger n is rejected.  The first call on a device
 * looks up that array's device address (with the device current); make it
 * before any stream capture.  All calls on a device share the array, so calls
 * whose work overlaps on the GPU race with each other: order them on one
 * stream or synchronise between them.  Nothing in the array needs to start
 * zeroed.  The looked-up address is kept for the library's lifetime, so a
 * cudaDeviceReset while the library stays loaded is not supported here. */
int wema_cuda_threshold_flat_noalloc(const float *d_x, size_t n, int threshold_form,
                                     float *d_thr, float *d_sum, void *cuda_stream);

/* ---- Batched streams: one frame tick over many streams ------------------
 * No counterpart in the reference (its CLI runs one stream per process).
 * A batch owns the device state of every stream added to it (IIR band-pass
 * streams, luma or colour, RGB24 frames in device memory) and advances a
 * chosen set of them by one frame per tick with one launch per kernel type
 * over all of them.  A stream's frames are bit-identical to what a
 * wema_cuda_session with the same config produces. */
typedef struct wema_cuda_batch wema_cuda_batch;

/* Device bytes one batched stream of this config holds (its admission cost). */
size_t wema_cuda_batch_stream_bytes(const wema_cuda_config *cfg);
int wema_cuda_batch_create(int device, int max_streams, wema_cuda_batch **out);
void wema_cuda_batch_destroy(wema_cuda_batch *b);
/* Allocates the stream's state; *id names it in later calls. */
int wema_cuda_batch_add(wema_cuda_batch *b, const wema_cuda_config *cfg, int *id);
/* Waits for the batch's work, then frees the stream's state. */
int wema_cuda_batch_remove(wema_cuda_batch *b, int id);
/* One frame of each of the n streams ids[k]: d_in_u8[k] (H x W x 3 RGB24 on
 * the device) -> d_out_u8[k].  Asynchronous: waits for wait_event (may be
 * NULL) before reading the inputs, records done_event (may be NULL) once every
 * output is written and no input is read any more.  A stream may appear once
 * per tick. */
int wema_cuda_batch_tick(wema_cuda_batch *b, const int *ids, const void *const *d_in_u8,
                         void *const *d_out_u8, int n, void *wait_event, void *done_event);
int wema_cuda_batch_sync(wema_cuda_batch *b);
/* The same tick with HOST frames (RGB24; pin them, e.g. with cudaHostAlloc,
 * for the copies to overlap): the tick's frames are copied into one of three
 * device staging sets the batch keeps (each a pair of arenas holding the
 * tick's frames back to back), the tick runs, the outputs are copied back -
 * so tick i-1's outputs go out while tick i+1's inputs come in and tick i
 * runs (the reference's async_io.c double buffering, on copy engines).  Frames
 * that lie back to back in host memory (in `ids` order) move in one copy;
 * many small copies in both directions at once run well below the host
 * link's rate.  Asynchronous: the copies in wait for wait_event (may be NULL)
 * and for the previous tick (see wema_cuda_batch_set_host_overlap); a host
 * buffer may be reused once
 * done_event (may be NULL) has completed, or after wema_cuda_batch_sync. */
int wema_cuda_batch_tick_host(wema_cuda_batch *b, const int *ids, const void *const *h_in_u8,
                              void *const *h_out_u8, int n, void *wait_event, void *done_event);
/* Per-stage device timing of the batched ticks (CUDA events on each stage's
 * stream, the WEMA_CUDA_STAGES order of wema_cuda_stage_times): times_ms[7]
 * receives the milliseconds summed over every timed tick, *ticks their
 * count.  Both wait for the batch. */
/* A steady tick - every listed stream past its first frame, stage timing
 * off - replays a CUDA graph of its launches, captured per parameter table
 * and set of launches, with the same kernels, parameters and results as the
 * launches themselves.  enable = 0: launch the kernels one by one, stage
 * after stage; default 1. */
int wema_cuda_batch_set_graphs(wema_cuda_batch *b, int enable);
/* Pipeline groups of a steady tick's graph (1..4, default 1): the tick's
 * streams are split into that many groups of about equal pixel count, and
 * group g's threshold, inverse and transfer run beside group g+1's forward,
 * threshold and inverse.  Results do not depend on it (on a B200 the
 * 48-stream mix ran fastest with one group). */
int wema_cuda_batch_set_groups(wema_cuda_batch *b, int groups);
/* enable = 1 (default): a host tick's copies in start as soon as their
 * staging set is free, beside the previous tick's kernels and copies out.
 * 0: they also wait for the previous tick to finish (measured slower on
 * B200 hosts: 9.7 against 12.7 Gpix-frames/s on a 48-stream mix). */
int wema_cuda_batch_set_host_overlap(wema_cuda_batch *b, int enable);
int wema_cuda_batch_set_timing(wema_cuda_batch *b, int enable);
int wema_cuda_batch_stage_times(wema_cuda_batch *b, double *times_ms, long long *ticks);
/* Snapshot / restore of one batched stream (as the session calls; a batched
 * stream's snapshot restores into a batched stream of the same config). */
size_t wema_cuda_batch_snapshot_bytes(wema_cuda_batch *b, int id);
int wema_cuda_batch_snapshot(wema_cuda_batch *b, int id, void *host, size_t cap);
int wema_cuda_batch_restore(wema_cuda_batch *b, int id, const void *host, size_t bytes);
/* Ticks issued, kernels launched, streams held. */
int wema_cuda_batch_stats(wema_cuda_batch *b, long long *ticks, long long *launches, int *live);
/* WEMA_CUDA_READ_THRESHOLD of a stream's last frame (waits for the batch). */
int wema_cuda_batch_read(wema_cuda_batch *b, int id, int what, int channel, void *host, size_t bytes);

/* ---- Served request loop -------------------------------------------------
 * No counterpart in the reference (a single-file CLI).  Camera-stream
 * sessions are admitted against a device-memory budget by their state bytes
 * (wema_cuda_batch_stream_bytes), queued first-in first-out while the budget
 * is full, and keep their state on the device until closed.  Frames submitted
 * at each stream's own rate are batched continuously: a dispatcher thread
 * puts the oldest pending frame of every live session into the next tick
 * whenever fewer than three ticks are in flight.  A session's outputs are
 * bit-identical to the same stream run alone. */
typedef struct wema_cuda_server wema_cuda_server;

enum {
    WEMA_CUDA_SESSION_QUEUED = 0,   /* waiting for budget */
    WEMA_CUDA_SESSION_LIVE = 1,     /* admitted: frames are accepted */
    WEMA_CUDA_SESSION_CLOSED = 2,   /* closed, state freed */
    WEMA_CUDA_SESSION_FAILED = 3    /* admission failed (device allocation) */
};

typedef struct {
    int state;                      /* WEMA_CUDA_SESSION_* */
    long long submitted, completed; /* frames accepted / whose output is written */
    long long dropped;              /* submissions refused (queued, or 8 pending) */
    size_t state_bytes;             /* the session's admission cost */
    double admission_wait_ms;       /* open -> admitted (-1 while queued) */
} wema_cuda_session_status;

typedef struct {
    double seconds;                 /* since creation or the last reset */
    long long ticks, frames, launches;
    double mpix_frames;             /* sum of W*H/1e6 over completed frames */
    float latency_p50_ms, latency_p99_ms, latency_max_ms;   /* submit -> output written */
    float admission_wait_p50_ms, admission_wait_max_ms;
    long long sessions_admitted;
    int sessions_live, sessions_queued;
    size_t bytes_used, budget_bytes;
    /* dispatcher: host time per tick issue, issue -> completion per tick,
     * longest session admission (state allocation) and retirement */
    float tick_host_ms_mean, tick_host_ms_max, tick_span_ms_mean, tick_span_ms_max;
    float admit_ms_max, retire_ms_max;
} wema_cuda_serve_stats;

int wema_cuda_server_create(int device, size_t budget_bytes, int max_streams, wema_cuda_server **out);
/* Waits for every issued tick, frees every session. */
void wema_cuda_server_destroy(wema_cuda_server *srv);
/* Fails when the config is invalid or its state alone exceeds the budget;
 * otherwise *sid names the session (admitted now or queued). */
int wema_cuda_server_open(wema_cuda_server *srv, const wema_cuda_config *cfg, int *sid);
/* One frame (H x W x 3 RGB24 on the device); both buffers must stay valid
 * until the session's completed count passes it.  0: accepted; 1: refused,
 * the session is still queued; 2: refused, 8 frames already pending. */
int wema_cuda_server_submit(wema_cuda_server *srv, int sid, const void *d_in_u8, void *d_out_u8);
/* Pending frames still run; then the state is freed and the queue advances. */
int wema_cuda_server_close(wema_cuda_server *srv, int sid);
int wema_cuda_server_poll(wema_cuda_server *srv, int sid, wema_cuda_session_status *st);
/* hold != 0: issue no new ticks (submitted frames collect; admission goes
 * on); 0 resumes.  For maintenance windows and for tests of tick mixing. */
int wema_cuda_server_hold(wema_cuda_server *srv, int hold);
/* Waits until no frame is pending or in flight and no session is queued. */
int wema_cuda_server_drain(wema_cuda_server *srv, int timeout_ms);
/* reset != 0 starts a new measurement window after filling *out. */
int wema_cuda_server_stats(wema_cuda_server *srv, int reset, wema_cuda_serve_stats *out);

/* Autotuner (no counterpart in the reference).  On this device it times
 *   - the temporal filter's step at 2, 4 and 8 coefficient positions per
 *     thread (a 2^23-position trial plane) and keeps the fastest (4, the
 *     default, unless another is more than 3% faster);
 *   - the batched guided filter's sweep at 64, 128 and 256 output rows per
 *     segment (a 3840x8640 trial frame) and keeps the fastest (64 until then);
 *   - the batched luma DWT level-0 kernels, forward and inverse, in nine
 *     variants each: CTAs per SM asked of the register allocator {1 (the
 *     compiler's choice), 3, 4} x lines lifted per warp at a time {2, 4, 8}
 *     (variant = 3 * index + index; a 3840x4320 trial frame, the forward
 *     with the temporal filter's step inside as steady batched ticks run it)
 *     and keeps the fastest of each (4x4 for both until then);
 * allocating ~950 MB for the trials (one at a time) and freeing it.  Every
 * later launch on the device uses the choices.  Returns the positions per
 * thread (or -1) and writes the timings to `report` (may be NULL; 1 KiB is
 * enough).  Results do not depend on any choice - each position's and each
 * pixel's arithmetic is the same - only speed does.  set / get fix or read a
 * choice directly (positions 2, 4 or 8; rows a multiple of 16 in 16..4096;
 * DWT variant 0..8, inverse = 0 forward, 1 inverse). */
int wema_cuda_autotune(int device, char *report, size_t cap);
int wema_cuda_set_iir_positions(int device, int positions);
int wema_cuda_get_iir_positions(int device);
int wema_cuda_set_guided_rows(int device, int rows);
int wema_cuda_get_guided_rows(int device);
int wema_cuda_set_dwt_variant(int device, int inverse, int variant);
int wema_cuda_get_dwt_variant(int device, int inverse);

/* Message of the last failure on this thread ("" if none). */
const char *wema_cuda_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WEMA_CUDA_H */
