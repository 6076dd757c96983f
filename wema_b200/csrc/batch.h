// batch.h - many video streams advanced one frame per tick, with one launch
// per kernel type and tick over every stream's (uneven) pyramid.
//
// Each stream keeps its own state (a Session holding one buffer set: pyramid,
// deltas, IIR state, threshold scratch and binade history) resident on the
// device.  A tick takes one frame of each listed stream and issues, on one
// CUDA stream, the same kernels as the per-stream path - forward DWT level 0
// (luma and colour streams apart), levels 1..3, threshold monoids and walk,
// the IIR filter (on a second CUDA stream, beside the threshold), inverse
// levels 3..1, inverse level 0 and the luma transfer - but each launch covers
// all streams: its grid is the concatenation of the streams' grids and a task
// map in device memory sends every block to its stream's parameters
// (multi.cuh).  The per-stream parameters and the maps of one tick are built on
// the host into one pinned table and copied with a single H2D copy; three
// tables rotate so the host can build tick t+1 while tick t runs.  The
// arithmetic is the per-stream path's, so a stream's frames are bit-identical
// alone and in any mix.
//
// A steady tick (every stream past its first frame) replays one CUDA graph
// of all its launches, captured per table and launch set.  The streams may be
// split into groups of about equal pixel count that run as a pipeline (group
// g's threshold beside group g+1's forward transform, its inverse beside group
// g+1's threshold, its transfer beside group g+1's inverse; threshold and
// inverse launches at the highest priority, the transfer at the lowest); one
// group is the default - on the 48-stream mix one group measured 2.19 ms per
// tick, two to four groups 2.32-2.36 ms (an earlier build: one graph 2.56 ms
// against three graphs per tick, with the transfer beside the next tick's
// forward, 2.65 ms).  The level-0 threshold monoids run on a branch of the
// graph beside the forward levels 1-3.  Other ticks
// (first frames, stage timing, graphs off) issue the stages in turn over all
// groups on streams: the luma transfer of tick t on its own lower-priority
// stream while tick t+1's forward, threshold and IIR run; tick t+1's inverse
// DWT, which rewrites the reconstructed luma the transfer reads, waits for it.
// The tick's done event follows its transfer.
//
// Supported per stream: IIR band-pass, luma (guided filter or Gaussian
// transfer) or colour, RGB24 frames in device memory.
#pragma once
#include <string.h>

#include <algorithm>
#include <array>
#include <mutex>
#include <new>
#include <vector>

#include "session.h"
#include "wema_cuda.h"

namespace wema {

namespace batch_detail {

// one batched launch being assembled: per-task parameter structs + grids
struct Launch {
    size_t elem = 0;
    std::vector<char> params;
    std::vector<int> gx, gy, nblk;
    unsigned total = 0;
    size_t params_off = 0, map_off = 0;   // device offsets in the tick's table
    bool any16 = false;                   // some task has FP16 planes (planes_fp16)
    void reset(size_t e) {
        elem = e;
        params.clear();
        gx.clear();
        gy.clear();
        nblk.clear();
        total = 0;
        any16 = false;
    }
    void add(const void* p, unsigned x, unsigned y, unsigned blocks) {
        if (blocks == 0) return;
        params.insert(params.end(), (const char*)p, (const char*)p + elem);
        gx.push_back((int)x);
        gy.push_back((int)y);
        nblk.push_back((int)blocks);
        total += blocks;
    }
    int n() const { return (int)gx.size(); }
};

enum {
    L_FWD0_LUMA, L_FWD0_COLOR, L_FWD1, L_FWD2, L_FWD3,
    L_THR_PART, L_THR_PREFIX, L_THR_MON, L_THR_WALK, L_THR16,
    L_THR_MON0,                         // monoids of the level-0 sub-chunks, split off
    L_IIR_PRESEED, L_IIR,
    L_INV3, L_INV2, L_INV1, L_INV0_LUMA, L_INV0_COLOR,
    L_XFER_GUIDED, L_XFER_GAUSS,
    L_COUNT
};

// timed stages (the per-stream path's order, WEMA_CUDA_STAGES)
enum { T_FWD0, T_FWD, T_THR, T_IIR, T_INV, T_INV0, T_XFER, T_COUNT };

}  // namespace batch_detail
using namespace batch_detail;

class Batch {
public:
    int device = 0;
    int max_streams = 0;
    std::vector<Session*> streams;        // by id; null when removed
    cudaStream_t st_main = nullptr, st_iir = nullptr, st_xfer = nullptr;
    // streams' state is allocated and zeroed on its own stream: a tick being
    // captured into a graph on st_main from another thread must not see it
    cudaStream_t st_alloc = nullptr;
    cudaEvent_t ev_fwd = nullptr, ev_iir = nullptr, ev_inv = nullptr, ev_xfer = nullptr;
    bool xfer_pending = false;            // ev_xfer marks a transfer on st_xfer tick t+1 must wait for
    static constexpr int NBUF = 3;
    struct Table {
        char* host = nullptr;
        char* host_dev = nullptr;         // host's device-mapped address
        char* dev = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;
        bool used = false;
        cudaEvent_t tev[T_COUNT][2] = {};  // stage start / end (timing on)
        bool timed = false;               // tev holds a tick not yet added to stage_ms
        // steady ticks replay a CUDA graph of their launches, one per table;
        // `sig` identifies the launches it holds
        cudaGraphExec_t g_tick = nullptr;
        std::vector<long long> sig;
        long long graph_launches = 0;   // kernels in one replay
    } tb[NBUF];
    bool use_graphs = true;
    // pipelined groups of a steady tick; the streams and events that build its graph
    static constexpr int MAXG = 4;
    int groups = 1;
    cudaStream_t cs_fwd = nullptr, cs_xfer = nullptr, cs_chain[MAXG] = {};
    cudaEvent_t ce_fork = nullptr, ce_f0[MAXG] = {}, ce_f[MAXG] = {}, ce_i[MAXG] = {}, ce_join[MAXG + 2] = {};
    bool timing = false;
    double stage_ms[T_COUNT] = {};
    long long ticks_timed = 0;

    // host-frame ticks: three device staging sets, each one arena for a tick's
    // frames in and one for its frames out (the tick's streams back to back),
    // copies on their own streams, so tick i-1's outputs go out while tick
    // i+1's inputs come in and tick i runs (async_io.c's double buffering, on
    // copy engines instead of threads; with two sets, tick i+1's copies in
    // would wait for tick i-1's copies out and the two directions would
    // alternate instead of overlapping).  Host frames that lie back to back
    // move in one copy.
    struct HostSet {
        cudaEvent_t h2d = nullptr, tick = nullptr, d2h = nullptr;
        bool used = false;
        uint8_t* din = nullptr;
        uint8_t* dout = nullptr;
        size_t cap = 0;                 // bytes of each arena
    } hs[3];
    cudaStream_t st_h2d = nullptr, st_d2h = nullptr;
    int hcur = 0;
    // on (the default): copies in wait only for their staging set's previous
    // tick (three ticks back), so they overlap the previous tick's kernels and
    // copies out - 12.7 Gpix-frames/s on the 48-stream mix on a B200 host,
    // against 9.7 with them after the previous tick (off).  This needs the
    // tick's parameter table to go in by a kernel: a table copy queued on
    // the copy engine behind the next tick's frames held each tick back
    bool host_overlap = true;
    int cur = 0;
    long long launches = 0;
    long long ticks = 0;
    Launch L[MAXG][L_COUNT];
    std::vector<char> image;

    ~Batch() {
        for (cudaStream_t st : {st_main, st_iir, st_xfer, st_h2d, st_d2h, st_alloc})
            if (st) cudaStreamSynchronize(st);
        for (HostSet& h : hs) {
            if (h.din) cudaFree(h.din);
            if (h.dout) cudaFree(h.dout);
        }
        for (Session* s : streams) delete s;
        for (Table& t : tb) {
            drop_graphs(t);
            if (t.host) cudaFreeHost(t.host);
            if (t.dev) cudaFree(t.dev);
            if (t.done) cudaEventDestroy(t.done);
            for (auto& p : t.tev)
                for (cudaEvent_t e : p)
                    if (e) cudaEventDestroy(e);
        }
        for (cudaStream_t st : {st_main, st_iir, st_xfer, st_h2d, st_d2h, st_alloc, cs_fwd, cs_xfer})
            if (st) cudaStreamDestroy(st);
        for (cudaStream_t st : cs_chain)
            if (st) cudaStreamDestroy(st);
        for (cudaEvent_t e : {ev_fwd, ev_iir, ev_inv, ev_xfer, ce_fork})
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ce_f)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ce_f0)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ce_i)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ce_join)
            if (e) cudaEventDestroy(e);
        for (HostSet& h : hs)
            for (cudaEvent_t e : {h.h2d, h.tick, h.d2h})
                if (e) cudaEventDestroy(e);
    }

    bool init(int dev, int max_n) {
        device = dev;
        max_streams = max_n;
        if (!ensure_device(dev)) return false;
        // streams' state comes from the device's stream-ordered pool; keep
        // freed state cached there for the next stream instead of returning it
        cudaMemPool_t pool;
        if (!cuda_ok(cudaDeviceGetDefaultMemPool(&pool, dev), "memory pool")) return false;
        uint64_t keep = ~0ull;
        if (!cuda_ok(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool"))
            return false;
        int lo = 0, hi = 0;
        if (!cuda_ok(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priorities")) return false;
        // the threshold (main stream) before the filter: its latency-bound
        // blocks take SMs first and the HBM-bound filter fills the rest
        const int mid = hi < lo ? hi + 1 : hi;
        if (!cuda_ok(cudaStreamCreateWithPriority(&st_main, cudaStreamNonBlocking, hi), "cudaStreamCreate") ||
            !cuda_ok(cudaStreamCreateWithPriority(&st_iir, cudaStreamNonBlocking, mid), "cudaStreamCreate"))
            return false;
        if (!cuda_ok(cudaStreamCreateWithPriority(&st_xfer, cudaStreamNonBlocking, lo), "cudaStreamCreate"))
            return false;
        for (cudaStream_t* st : {&st_h2d, &st_d2h, &st_alloc})
            if (!cuda_ok(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "cudaStreamCreate"))
                return false;
        // graph building: forward launches at the middle priority, threshold and
        // inverse chains at the highest, the transfer at the lowest (the graph
        // keeps each launch's priority)
        if (!cuda_ok(cudaStreamCreateWithPriority(&cs_fwd, cudaStreamNonBlocking, mid), "cudaStreamCreate") ||
            !cuda_ok(cudaStreamCreateWithPriority(&cs_xfer, cudaStreamNonBlocking, lo), "cudaStreamCreate"))
            return false;
        for (cudaStream_t& st : cs_chain)
            if (!cuda_ok(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi), "cudaStreamCreate"))
                return false;
        for (cudaEvent_t* e : {&ce_fork})
            if (!cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate")) return false;
        for (int g = 0; g < MAXG; g++)
            if (!cuda_ok(cudaEventCreateWithFlags(&ce_f[g], cudaEventDisableTiming), "cudaEventCreate") ||
                !cuda_ok(cudaEventCreateWithFlags(&ce_f0[g], cudaEventDisableTiming), "cudaEventCreate") ||
                !cuda_ok(cudaEventCreateWithFlags(&ce_i[g], cudaEventDisableTiming), "cudaEventCreate"))
                return false;
        for (cudaEvent_t& e : ce_join)
            if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")) return false;
        for (HostSet& h : hs)
            for (cudaEvent_t* e : {&h.h2d, &h.tick, &h.d2h})
                if (!cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate"))
                    return false;
        for (cudaEvent_t* e : {&ev_fwd, &ev_iir, &ev_inv, &ev_xfer})
            if (!cuda_ok(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate"))
                return false;
        for (Table& t : tb)
            if (!cuda_ok(cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming), "cudaEventCreate"))
                return false;
        return true;
    }

    int live() const {
        int n = 0;
        for (Session* s : streams) n += s != nullptr;
        return n;
    }

    int add(const wema_cuda_config& c) {
        if (live() >= max_streams) { set_error("batch holds %d streams already", max_streams); return -1; }
        Session* s = make(c);
        return s ? insert(s) : -1;
    }

    // A stream's state, allocated and zeroed on the allocation stream, which
    // this call then waits for (so the state is ready for any later tick); the
    // batch itself is untouched, so another host thread may call this while
    // ticks are issued (then insert() it from the ticking thread).
    Session* make(const wema_cuda_config& c) {
        if (!c.use_iir) { set_error("batched streams use the IIR filter (use_iir = 1)"); return nullptr; }
        if (c.device != device) { set_error("stream device %d differs from the batch's %d", c.device, device); return nullptr; }
        Session* s = new (std::nothrow) Session();
        if (!s) { set_error("out of host memory"); return nullptr; }
        if (!s->init(c, 1, st_alloc) || !cuda_ok(cudaStreamSynchronize(st_alloc), "state allocation")) {
            delete s;
            return nullptr;
        }
        return s;
    }

    // takes ownership of a made stream; its id
    int insert(Session* s) {
        if (live() >= max_streams) {
            delete s;
            set_error("batch holds %d streams already", max_streams);
            return -1;
        }
        for (size_t i = 0; i < streams.size(); i++)
            if (!streams[i]) { streams[i] = s; return (int)i; }
        streams.push_back(s);
        return (int)streams.size() - 1;
    }

    // wait = false: the caller knows the stream's last tick has completed
    bool remove(int id, bool wait = true) {
        if (id < 0 || id >= (int)streams.size() || !streams[id]) { set_error("no stream %d", id); return false; }
        if (wait && !sync()) return false;
        delete streams[id];
        streams[id] = nullptr;
        return true;
    }

    // adds a completed table's stage times to the totals
    bool collect(Table& t) {
        if (!t.timed) return true;
        for (int k = 0; k < T_COUNT; k++) {
            float ms = 0.f;
            if (!cuda_ok(cudaEventElapsedTime(&ms, t.tev[k][0], t.tev[k][1]), "stage time")) return false;
            stage_ms[k] += ms;
        }
        ticks_timed++;
        t.timed = false;
        return true;
    }

    // totals over every timed tick (waits for the batch)
    bool stage_times(double* ms, long long* n) {
        if (!sync()) return false;
        for (Table& t : tb)
            if (!collect(t)) return false;
        for (int k = 0; k < T_COUNT; k++) ms[k] = stage_ms[k];
        *n = ticks_timed;
        return true;
    }


    bool sync() {
        if (!cuda_ok(cudaStreamSynchronize(st_h2d), "sync")) return false;
        if (!cuda_ok(cudaStreamSynchronize(st_iir), "sync")) return false;
        if (!cuda_ok(cudaStreamSynchronize(st_main), "sync")) return false;
        if (!cuda_ok(cudaStreamSynchronize(st_xfer), "sync")) return false;
        return cuda_ok(cudaStreamSynchronize(st_d2h), "sync");
    }

    // One tick with host frames (RGB24, pinned for the copies to be
    // asynchronous): copies in on st_h2d, the tick, copies out on st_d2h.
    // `done` (may be null) is recorded once every output is in host memory.
    bool tick_host(const int* ids, const uint8_t* const* h_in, uint8_t* const* h_out, int n,
                   cudaEvent_t wait, cudaEvent_t done) {
        HostSet& S = hs[hcur];
        std::vector<size_t> off(n + 1, 0);
        for (int k = 0; k < n; k++) {
            const int id = ids[k];
            if (id < 0 || id >= (int)streams.size() || !streams[id]) { set_error("no stream %d", id); return false; }
            if (!h_in[k] || !h_out[k]) { set_error("stream %d: null frame", id); return false; }
            const size_t fb = 3 * (size_t)streams[id]->g.pixels;
            off[k + 1] = off[k] + ((fb + 255) & ~(size_t)255);   // 256-byte aligned frames
        }
        // this set was last used three ticks ago: its tick has read the inputs and
        // its outputs have gone out before they are overwritten
        if (S.used && (!cuda_ok(cudaStreamWaitEvent(st_h2d, S.tick, 0), "stream wait") ||
                       !cuda_ok(cudaStreamWaitEvent(st_h2d, S.d2h, 0), "stream wait")))
            return false;
        const HostSet& P = hs[(hcur + 2) % 3];   // the previous tick's set
        if (!host_overlap && P.used && !cuda_ok(cudaStreamWaitEvent(st_h2d, P.tick, 0), "stream wait"))
            return false;
        if (wait && !cuda_ok(cudaStreamWaitEvent(st_h2d, wait, 0), "stream wait")) return false;
        if (off[n] > S.cap) {                  // grow the set's arenas, in stream order after its last use
            if (S.din) cudaFreeAsync(S.din, st_h2d);
            if (S.dout) cudaFreeAsync(S.dout, st_h2d);
            S.din = S.dout = nullptr;
            S.cap = 0;
            if (!cuda_ok(cudaMallocAsync((void**)&S.din, off[n], st_h2d), "cudaMallocAsync(host staging)"))
                return false;
            if (!cuda_ok(cudaMallocAsync((void**)&S.dout, off[n], st_h2d), "cudaMallocAsync(host staging)")) {
                cudaFreeAsync(S.din, st_h2d);
                S.din = nullptr;
                return false;
            }
            S.cap = off[n];
        }
        std::vector<const uint8_t*> din(n);
        std::vector<uint8_t*> dout(n);
        for (int k = 0; k < n; k++) {
            din[k] = S.din + off[k];
            dout[k] = S.dout + off[k];
        }
        // runs of frames contiguous on both sides move as one copy
        auto copies = [&](bool in, cudaStream_t st) {
            for (int k = 0; k < n;) {
                const int k0 = k;
                size_t len = 3 * (size_t)streams[ids[k]]->g.pixels;
                // frame k+1 joins while it follows the run directly in the arena (no
                // alignment gap) and in host memory
                while (k + 1 < n && off[k + 1] - off[k0] == len &&
                       (in ? h_in[k + 1] == h_in[k0] + len : h_out[k + 1] == h_out[k0] + len)) {
                    k++;
                    len += 3 * (size_t)streams[ids[k]]->g.pixels;
                }
                const bool ok = in ? cuda_ok(cudaMemcpyAsync((void*)din[k0], h_in[k0], len, cudaMemcpyHostToDevice, st),
                                             "copy in")
                                   : cuda_ok(cudaMemcpyAsync(h_out[k0], dout[k0], len, cudaMemcpyDeviceToHost, st),
                                             "copy out");
                if (!ok) return false;
                k++;
            }
            return true;
        };
        if (!copies(true, st_h2d)) return false;
        if (!cuda_ok(cudaEventRecord(S.h2d, st_h2d), "event record")) return false;
        if (!tick(ids, din.data(), dout.data(), n, S.h2d, S.tick)) return false;
        if (!cuda_ok(cudaStreamWaitEvent(st_d2h, S.tick, 0), "stream wait")) return false;
        if (!copies(false, st_d2h)) return false;
        if (!cuda_ok(cudaEventRecord(S.d2h, st_d2h), "event record")) return false;
        if (done && !cuda_ok(cudaEventRecord(done, st_d2h), "event record")) return false;
        S.used = true;
        hcur = (hcur + 1) % 3;
        return true;
    }

    static void drop_graphs(Table& t) {
        if (t.g_tick) {
            cudaGraphExecDestroy(t.g_tick);
            t.g_tick = nullptr;
        }
        t.sig.clear();
    }

    // records what `issue` launches on `st` as a graph (nothing runs)
    template <class F>
    bool capture(cudaStream_t st, cudaGraphExec_t* out, F issue) {
        if (!cuda_ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture")) return false;
        const bool ok = issue();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (!ok || !cuda_ok(e, "end capture")) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        const bool inst = cuda_ok(cudaGraphInstantiateWithFlags(out, g, cudaGraphInstantiateFlagUseNodePriority),
                                  "graph instantiate");
        cudaGraphDestroy(g);
        return inst;
    }

    // the table image: every launch's parameter array, then its task map
    size_t put(const void* p, size_t n) {
        size_t off = (image.size() + 15) & ~(size_t)15;
        image.resize(off + n);
        if (n) memcpy(image.data() + off, p, n);
        return off;
    }
    void emit(Launch& l) {
        if (l.n() == 0) return;
        l.params_off = put(l.params.data(), l.params.size());
        const int n = l.n();
        std::vector<int> map(3 * n + 2);
        map[0] = n;
        int start = 0;
        for (int i = 0; i < n; i++) {
            map[1 + i] = start;
            start += l.nblk[i];
        }
        map[1 + n] = start;
        for (int i = 0; i < n; i++) {
            map[n + 2 + i] = l.gx[i];
            map[2 * n + 2 + i] = l.gy[i];
        }
        l.map_off = put(map.data(), map.size() * sizeof(int));
    }

    bool tick(const int* ids, const uint8_t* const* in, uint8_t* const* out, int n, cudaEvent_t wait,
              cudaEvent_t done) {
        for (int k = 0; k < n; k++) {
            if (ids[k] < 0 || ids[k] >= (int)streams.size() || !streams[ids[k]]) {
                set_error("no stream %d", ids[k]);
                return false;
            }
            if (!in[k] || !out[k]) { set_error("stream %d: null frame", ids[k]); return false; }
            for (int q = 0; q < k; q++)
                if (ids[q] == ids[k]) { set_error("stream %d listed twice in one tick", ids[k]); return false; }
        }
        for (auto& LG : L) {
            LG[L_FWD0_LUMA].reset(sizeof(FwdLevelParams));
            LG[L_FWD0_COLOR].reset(sizeof(FwdLevelParams));
            for (int l = 1; l <= 3; l++) LG[L_FWD0_COLOR + l].reset(sizeof(FwdLevelParams));
            for (int k = L_THR_PART; k <= L_THR_MON0; k++) LG[k].reset(thr_args_bytes());
            LG[L_IIR_PRESEED].reset(iir_args_bytes());
            LG[L_IIR].reset(iir_args_bytes());
            for (int k = L_INV3; k <= L_INV0_COLOR; k++) LG[k].reset(sizeof(InvLevelParams));
            LG[L_XFER_GUIDED].reset(sizeof(TransferParams));
            LG[L_XFER_GAUSS].reset(sizeof(TransferParams));
        }
        std::vector<char> targs(thr_args_bytes()), iargs(iir_args_bytes());

        // streams largest first: every launch lists its tasks in that order, so
        // the blocks of the longest tasks (a 4K stream's threshold walk lanes)
        // start in the first wave instead of trailing the launch; the pipeline's
        // groups take the streams in the same order, each to the group with the
        // fewest pixels so far
        const int G = std::max(1, std::min(groups, n));
        std::vector<int> grp(n, 0), order(n);
        for (int k = 0; k < n; k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return streams[ids[a]]->g.pixels > streams[ids[b]]->g.pixels;
        });
        {
            long long load[MAXG] = {};
            for (int k : order) {
                int best = 0;
                for (int g = 1; g < G; g++)
                    if (load[g] < load[best]) best = g;
                grp[k] = best;
                load[best] += streams[ids[k]]->g.pixels;
            }
        }

        for (const int k : order) {
            Session& S = *streams[ids[k]];
            Launch* const LK = L[grp[k]];
            const Geom& g = S.g;
            const int LV = g.levels, nch = S.nch;
            Slot& q = S.slot[0];
            // ---- forward DWT
            for (int l = 0; l < LV; l++) {
                FwdLevelParams p{};
                p.iw = g.in_w[l];
                p.ih = g.in_h[l];
                p.sw = g.sw[l];
                p.sh = g.sh[l];
                p.n = g.n[l];
                p.vec_end = vec_cover(g.pixels);
                if (l == 0) p.src_u8 = in[k];
                else
                    for (int c = 0; c < nch; c++) p.src_planes[c] = q.ll[c][l - 1];
                const bool h = S.cfg.planes_fp16;
                for (int c = 0; c < nch; c++) {
                    p.coef[c] = plane_at(q.coef[c], g.uoff[l], h);
                    p.prev[c] = l > 0 ? plane_at(q.coef[c], g.uoff[l - 1], h) : nullptr;
                    p.ll_out[c] = q.ll[c][l];
                }
                p.h16 = h;
                p.prev_n = l > 0 ? g.n[l - 1] : 0;
                if (S.frames_processed > 0) S.fill_temporal(p, l);   // the filter's step inside the transform
                unsigned gx, gy;
                Launch& lf = LK[l == 0 ? (nch == 3 ? L_FWD0_COLOR : L_FWD0_LUMA) : L_FWD0_COLOR + l];
                const unsigned b = dwt_fwd_grid(p, l == 0 ? 1 : nch, gx, gy);
                lf.add(&p, gx, gy, b);
                lf.any16 |= h;
            }
            // ---- threshold
            PyrView views[3];
            for (int c = 0; c < nch; c++) views[c] = S.view(0, c);
            unsigned grids[5][2];
            if (!cuda_ok(thr_args_fill(targs.data(), views, nch, S.thr_s, q.thr, q.thr + 4,
                                       S.cfg.threshold_form, S.thr_hist ? 1 : 0, grids),
                         "threshold setup"))
                return false;
            // with a binade history the monoids of the sub-chunks wholly in level 0
            // go in a launch of their own, which a steady tick runs beside the
            // forward transform's levels 1-3
            const int split = S.thr_hist && !S.cfg.planes_fp16 ? thr_level0_subchunks(views[0]) : 0;
            for (int st = 0; st < 5; st++) {
                if ((st == 4) != (S.cfg.planes_fp16 != 0)) continue;   // FP16 planes: one kernel
                if (st < 2 && S.thr_hist) continue;   // partial sums + prefix: first frame only
                if (st == 2 && split > 0) {
                    std::vector<char> part(targs);
                    const unsigned b0 = thr_args_monoid_part(part.data(), 0, split);
                    LK[L_THR_MON0].add(part.data(), b0, grids[st][1], b0 * grids[st][1]);
                    const unsigned b1 = thr_args_monoid_part(part.data(), split, -1);
                    LK[L_THR_MON].add(part.data(), b1, grids[st][1], b1 * grids[st][1]);
                    continue;
                }
                LK[L_THR_PART + st].add(targs.data(), grids[st][0], grids[st][1],
                                       grids[st][0] * grids[st][1]);
            }
            // ---- IIR: a stream's first frame takes the preseed and the filter as
            // launches of their own; after it the forward transform runs the step
            const bool first = S.frames_processed == 0;
            for (int c = 0; first && c < nch; c++) {
                const unsigned b = iir_args_fill(iargs.data(), S.ip, q.coef[c], S.state[c], S.cfg.iir_state_fp64, q.delta[c],
                                                 S.warmup);
                LK[L_IIR_PRESEED].add(iargs.data(), b, 1, b);
                LK[L_IIR].add(iargs.data(), b, 1, b);
            }
            // ---- inverse DWT (+ colour output) and the luma transfer
            const float amp = fade_amp(S.cfg.amp_factor, first ? S.warmup : S.frames_processed, S.warmup);
            q.alpha[0] = amp;
            q.alpha[1] = q.alpha[2] = amp * 0.5f;
            for (int l = LV - 1; l >= 0; l--) {
                InvLevelParams iq{};
                iq.ow = g.in_w[l];
                iq.oh = g.in_h[l];
                iq.sw = g.sw[l];
                iq.sh = g.sh[l];
                iq.n = g.n[l];
                iq.thr = q.thr;
                iq.h16 = S.cfg.planes_fp16;
                iq.out16 = S.cfg.planes_fp16 && l == 0;
                for (int c = 0; c < nch; c++) {
                    iq.ll[c] = (l == LV - 1) ? q.ll[c][LV - 1] : q.rec[c][l + 1];
                    iq.coef[c] = plane_at(q.coef[c], g.uoff[l], iq.h16);
                    iq.delta[c] = plane_at(q.delta[c], g.uoff[l], iq.h16);
                    iq.alpha[c] = l == 0 ? q.alpha[c] * 0.5f : q.alpha[c];
                    iq.out_planes[c] = (l > 0 || nch == 1) ? q.rec[c][l] : nullptr;
                }
                unsigned gx, gy;
                if (l == 0 && nch == 3) iq.out_u8 = out[k];
                Launch& li = LK[l == 0 ? (nch == 3 ? L_INV0_COLOR : L_INV0_LUMA) : L_INV1 - (l - 1)];
                const unsigned b = dwt_inv_grid(iq, l == 0 && nch == 3 ? 1 : nch, gx, gy);
                li.add(&iq, gx, gy, b);
                li.any16 |= iq.h16 != 0;
            }
            if (nch == 1) {
                TransferParams tp{};
                tp.w = g.w;
                tp.h = g.h;
                tp.vec_end = vec_cover(g.pixels);
                tp.src_u8 = in[k];
                tp.gray_out = q.rec[0][0];
                tp.out_u8 = out[k];
                tp.edge_aware = S.cfg.edge_aware;
                tp.h16 = S.cfg.planes_fp16;
                unsigned gx, gy;
                const unsigned b = transfer_grid(tp, gx, gy);
                LK[tp.edge_aware ? L_XFER_GUIDED : L_XFER_GAUSS].add(&tp, gx, gy, b);
            }
        }
        // ---- the table image, its buffer, one H2D copy
        image.clear();
        for (auto& LG : L)
            for (Launch& l : LG) emit(l);
        Table& t = tb[cur];
        if (t.used && !cuda_ok(cudaEventSynchronize(t.done), "table reuse")) return false;
        if (!collect(t)) return false;
        if (image.size() > t.cap) {
            if (t.host) cudaFreeHost(t.host);
            if (t.dev) cudaFree(t.dev);
            t.host = nullptr;
            t.dev = nullptr;
            t.cap = 0;
            const size_t cap = std::max<size_t>(image.size() * 2, 1 << 16);
            if (!cuda_ok(cudaHostAlloc(&t.host, cap, cudaHostAllocMapped), "cudaHostAlloc(table)")) return false;
            if (!cuda_ok(cudaHostGetDevicePointer((void**)&t.host_dev, t.host, 0), "table mapping")) return false;
            if (!cuda_ok(cudaMalloc(&t.dev, cap), "cudaMalloc(table)")) return false;
            t.cap = cap;
        }
        memcpy(t.host, image.data(), image.size());
        if (wait && !cuda_ok(cudaStreamWaitEvent(st_main, wait, 0), "stream wait")) return false;
        // the table by a kernel, not a copy engine: with host ticks the H2D engine
        // may be busy with the next tick's frames
        launches += 1;
        if (!cuda_ok(launch_table_copy(t.dev, t.host_dev, image.size(), st_main), "table copy")) return false;
        auto P = [&](int g, int k) { return (const void*)(t.dev + L[g][k].params_off); };
        auto M = [&](int g, int k) { return (const int*)(t.dev + L[g][k].map_off); };
        auto ok = [&](cudaError_t e, const char* what) {
            launches += 1;
            return cuda_ok(e, what);
        };
        auto go = [&](int g, int k, auto fn, const char* what) {
            if (L[g][k].n() == 0) return true;
            return ok(fn(), what);
        };
        auto mark = [&](int stage, int end, cudaStream_t st) {
            return !timing || cuda_ok(cudaEventRecord(t.tev[stage][end], st), "event record");
        };
        if (timing && !t.tev[0][0])
            for (auto& p : t.tev)
                for (cudaEvent_t& e : p)
                    if (!cuda_ok(cudaEventCreate(&e), "cudaEventCreate")) return false;

        // the stages of one group on one stream
        auto fwd0 = [&](int g, cudaStream_t st) {
            return go(g, L_FWD0_LUMA, [&] { return launch_dwt_fwd_multi(kSrcRgbU8, 1, (const FwdLevelParams*)P(g, L_FWD0_LUMA), M(g, L_FWD0_LUMA), L[g][L_FWD0_LUMA].total, L[g][L_FWD0_LUMA].any16, st); }, "forward DWT") &&
                   go(g, L_FWD0_COLOR, [&] { return launch_dwt_fwd_multi(kSrcRgbU8, 3, (const FwdLevelParams*)P(g, L_FWD0_COLOR), M(g, L_FWD0_COLOR), L[g][L_FWD0_COLOR].total, L[g][L_FWD0_COLOR].any16, st); }, "forward DWT");
        };
        auto fwdl = [&](int g, cudaStream_t st) {
            for (int k = L_FWD1; k <= L_FWD3; k++)
                if (!go(g, k, [&] { return launch_dwt_fwd_multi(kSrcPlanes, 1, (const FwdLevelParams*)P(g, k), M(g, k), L[g][k].total, L[g][k].any16, st); }, "forward DWT"))
                    return false;
            return true;
        };
        // threshold launches in order: partials, prefix, level-0 monoids, other
        // monoids, walk, FP16 sum (a launch with no tasks is skipped); thr_a / thr_b
        // are the parts before and after the forward transform's levels 1-3
        auto thr_range = [&](int g, cudaStream_t st, int i0, int i1) {
            static const int kind[6] = {L_THR_PART, L_THR_PREFIX, L_THR_MON0, L_THR_MON, L_THR_WALK, L_THR16};
            static const int stage[6] = {0, 1, 2, 2, 3, 4};
            for (int i = i0; i < i1; i++) {
                const int k = kind[i];
                if (!go(g, k, [&] { return launch_threshold_multi(stage[i], P(g, k), M(g, k), L[g][k].total, st); }, "threshold"))
                    return false;
            }
            return true;
        };
        auto thr = [&](int g, cudaStream_t st) { return thr_range(g, st, 0, 6); };
        auto thr_a = [&](int g, cudaStream_t st) { return thr_range(g, st, 2, 3); };
        auto thr_b = [&](int g, cudaStream_t st) { return thr_range(g, st, 0, 2) && thr_range(g, st, 3, 6); };
        auto iir = [&](int g, cudaStream_t st) {
            return go(g, L_IIR_PRESEED, [&] { return launch_iir_multi(P(g, L_IIR_PRESEED), M(g, L_IIR_PRESEED), L[g][L_IIR_PRESEED].total, 1, st); }, "IIR preseed") &&
                   go(g, L_IIR, [&] { return launch_iir_multi(P(g, L_IIR), M(g, L_IIR), L[g][L_IIR].total, 0, st); }, "IIR");
        };
        auto invl = [&](int g, cudaStream_t st) {
            for (int k = L_INV3; k <= L_INV1; k++)
                if (!go(g, k, [&] { return launch_dwt_inv_multi(1, kOutPlanes, (const InvLevelParams*)P(g, k), M(g, k), L[g][k].total, L[g][k].any16, st); }, "inverse DWT"))
                    return false;
            return true;
        };
        auto inv0 = [&](int g, cudaStream_t st) {
            return go(g, L_INV0_LUMA, [&] { return launch_dwt_inv_multi(1, kOutPlanes, (const InvLevelParams*)P(g, L_INV0_LUMA), M(g, L_INV0_LUMA), L[g][L_INV0_LUMA].total, L[g][L_INV0_LUMA].any16, st); }, "inverse DWT") &&
                   go(g, L_INV0_COLOR, [&] { return launch_dwt_inv_multi(3, kOutRgb, (const InvLevelParams*)P(g, L_INV0_COLOR), M(g, L_INV0_COLOR), L[g][L_INV0_COLOR].total, L[g][L_INV0_COLOR].any16, st); }, "inverse DWT");
        };
        auto xfer = [&](int g, cudaStream_t st) {
            return go(g, L_XFER_GUIDED, [&] { return launch_transfer_multi(1, (const TransferParams*)P(g, L_XFER_GUIDED), M(g, L_XFER_GUIDED), L[g][L_XFER_GUIDED].total, st); }, "luma transfer") &&
                   go(g, L_XFER_GAUSS, [&] { return launch_transfer_multi(0, (const TransferParams*)P(g, L_XFER_GAUSS), M(g, L_XFER_GAUSS), L[g][L_XFER_GAUSS].total, st); }, "luma transfer");
        };
        // a stage over every group in turn, between its timing marks
        auto all = [&](auto stage, int tstage, cudaStream_t st) {
            if (!mark(tstage, 0, st)) return false;
            for (int g = 0; g < G; g++)
                if (!stage(g, st)) return false;
            return mark(tstage, 1, st);
        };
        // The steady tick's pipeline, issued on st_main while it is captured:
        // forward transforms group after group on cs_fwd; per group a chain
        // (threshold, then inverse after the previous group's) on cs_chain[g];
        // transfers group after group on cs_xfer; all joined back to st_main.
        auto pipeline = [&] {
            if (!cuda_ok(cudaEventRecord(ce_fork, st_main), "event record") ||
                !cuda_ok(cudaStreamWaitEvent(cs_fwd, ce_fork, 0), "stream wait"))
                return false;
            for (int g = 0; g < G; g++)
                if (!fwd0(g, cs_fwd) || !cuda_ok(cudaEventRecord(ce_f0[g], cs_fwd), "event record") ||
                    !fwdl(g, cs_fwd) || !cuda_ok(cudaEventRecord(ce_f[g], cs_fwd), "event record"))
                    return false;
            for (int g = 0; g < G; g++) {
                cudaStream_t cs = cs_chain[g];
                // level-0 monoids beside levels 1-3 of the forward transform
                if (!cuda_ok(cudaStreamWaitEvent(cs, ce_f0[g], 0), "stream wait") || !thr_a(g, cs)) return false;
                if (!cuda_ok(cudaStreamWaitEvent(cs, ce_f[g], 0), "stream wait") || !thr_b(g, cs)) return false;
                if (g > 0 && !cuda_ok(cudaStreamWaitEvent(cs, ce_i[g - 1], 0), "stream wait")) return false;
                if (!invl(g, cs) || !inv0(g, cs) || !cuda_ok(cudaEventRecord(ce_i[g], cs), "event record"))
                    return false;
            }
            for (int g = 0; g < G; g++)
                if (!cuda_ok(cudaStreamWaitEvent(cs_xfer, ce_i[g], 0), "stream wait") || !xfer(g, cs_xfer))
                    return false;
            int nj = 0;
            auto join = [&](cudaStream_t st) {
                return cuda_ok(cudaEventRecord(ce_join[nj], st), "event record") &&
                       cuda_ok(cudaStreamWaitEvent(st_main, ce_join[nj++], 0), "stream wait");
            };
            if (!join(cs_fwd) || !join(cs_xfer)) return false;
            for (int g = 0; g < G; g++)
                if (!join(cs_chain[g])) return false;
            return true;
        };

        bool first_frames = false;
        for (int g = 0; g < G; g++)
            first_frames |= L[g][L_IIR].n() || L[g][L_IIR_PRESEED].n() || L[g][L_THR_PART].n() || L[g][L_THR_PREFIX].n();
        const bool steady = use_graphs && !timing && !first_frames;
        if (steady) {
            // what the graph holds: the table, every launch's blocks and offsets,
            // the device's kernel variants
            std::vector<long long> sig = {(long long)(uintptr_t)t.dev, dwt_variant(device, 0), dwt_variant(device, 1), G};
            for (int g = 0; g < G; g++)
                for (const Launch& l : L[g]) {
                    sig.push_back(l.total);
                    sig.push_back((long long)l.params_off);
                    sig.push_back((long long)l.map_off);
                    sig.push_back(l.any16);
                }
            if (sig != t.sig) {
                drop_graphs(t);
                const long long before = launches;
                if (!capture(st_main, &t.g_tick, pipeline)) {
                    drop_graphs(t);
                    return false;
                }
                t.graph_launches = launches - before;
                launches = before;
                t.sig = sig;
            }
            launches += t.graph_launches;
            // a transfer outside the graphs (an earlier unsteady tick's, on st_xfer) may still
            // read its reconstructed luma; a steady tick's transfer is in st_main's order
            if (xfer_pending && !cuda_ok(cudaStreamWaitEvent(st_main, ev_xfer, 0), "stream wait")) return false;
            if (!cuda_ok(cudaGraphLaunch(t.g_tick, st_main), "graph launch")) return false;
            if (!cuda_ok(cudaEventRecord(ev_inv, st_main), "event record")) return false;
            if (!cuda_ok(cudaStreamWaitEvent(st_xfer, ev_inv, 0), "stream wait")) return false;
        } else {
            // forward, then the filter (first frames) beside the threshold
            if (!all(fwd0, T_FWD0, st_main) || !all(fwdl, T_FWD, st_main)) return false;
            if (!cuda_ok(cudaEventRecord(ev_fwd, st_main), "event record")) return false;
            if (!all(thr, T_THR, st_main)) return false;
            if (!cuda_ok(cudaStreamWaitEvent(st_iir, ev_fwd, 0), "stream wait")) return false;
            if (!all(iir, T_IIR, st_iir)) return false;
            if (!cuda_ok(cudaEventRecord(ev_iir, st_iir), "event record")) return false;
            if (!cuda_ok(cudaStreamWaitEvent(st_main, ev_iir, 0), "stream wait")) return false;
            // the previous tick's transfer still reads its reconstructed luma
            if (xfer_pending && !cuda_ok(cudaStreamWaitEvent(st_main, ev_xfer, 0), "stream wait")) return false;
            if (!all(invl, T_INV, st_main) || !all(inv0, T_INV0, st_main)) return false;
            // the transfer on its own stream, so the next tick's forward half overlaps it
            if (!cuda_ok(cudaEventRecord(ev_inv, st_main), "event record")) return false;
            if (!cuda_ok(cudaStreamWaitEvent(st_xfer, ev_inv, 0), "stream wait")) return false;
            if (!all(xfer, T_XFER, st_xfer)) return false;
        }
        if (!cuda_ok(cudaEventRecord(ev_xfer, st_xfer), "event record")) return false;
        // only a transfer issued on st_xfer makes the next tick wait for ev_xfer (a
        // steady tick's transfer is in st_main's order already)
        xfer_pending = !steady;
        t.timed = timing;
        if (!cuda_ok(cudaEventRecord(t.done, st_xfer), "event record")) return false;
        if (done && !cuda_ok(cudaEventRecord(done, st_xfer), "event record")) return false;
        t.used = true;
        cur = (cur + 1) % NBUF;
        ticks++;

        // per-stream frame bookkeeping, as the per-stream path does it
        for (int k = 0; k < n; k++) {
            Session& S = *streams[ids[k]];
            if (S.frames_processed == 0) S.frames_processed = S.warmup;
            S.frames_processed++;
            S.thr_hist = true;
            S.slot[0].valid = true;
            S.last_slot = 0;
            S.frames_run++;
        }
        return true;
    }
};

}  // namespace wema
