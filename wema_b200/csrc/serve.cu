// serve.cu - the served request loop: camera-stream sessions admitted against
// a device-memory budget, their frames batched continuously into ticks.
//
// A session is opened with its stream config.  Its admission cost is the
// device state a batched stream of that config holds (pyramid, deltas, biquad
// state, threshold scratch: Session::bytes_for); it is admitted at once when
// that fits the budget beside the live sessions, else it waits in a FIFO queue
// and is admitted as closing sessions free memory.  Clients submit frames
// (device RGB24 in / out) at their own rates.  One dispatcher thread owns the
// Batch: whenever fewer than three ticks are in flight it takes the oldest
// pending frame of every live session into one tick, so a frame that arrives
// while the device is busy joins the next tick (continuous batching) and
// consecutive ticks overlap on the device.  A second thread allocates admitted
// sessions' state, so the dispatcher never waits for an allocation.  A host
// callback stamps each tick's completion; a frame's latency is completion
// minus submission.
//
// A session's frames run in submission order through its own device state,
// the same kernels and arithmetic as the stream alone, so its outputs do not
// depend on which other sessions share its ticks.
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <string>
#include <thread>

#include "batch.h"

namespace wema {

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

float pct(std::vector<float> v, double q) {
    if (v.empty()) return 0.f;
    const size_t k = std::min(v.size() - 1, (size_t)floor(q * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

class Server {
public:
    struct Frame {
        const uint8_t* in;
        uint8_t* out;
        double t_submit;
    };
    struct Sess {
        wema_cuda_config cfg{};
        size_t bytes = 0;
        int state = WEMA_CUDA_SESSION_QUEUED;
        int bid = -1;                      // stream id in the batch
        double t_open = 0, t_admit = 0;
        std::deque<Frame> pending;
        long long submitted = 0, completed = 0, inflight = 0, dropped = 0;
        bool closing = false;
        std::string err;
    };
    struct Tick {
        Server* srv;
        std::vector<int> sids;
        std::vector<double> t_submit;
        double t_issue = 0, t_done = -1;
        cudaEvent_t ev = nullptr;          // recorded when the tick's outputs are written
    };
    // completion events for ticks, reused; the dispatcher polls them (no host
    // callback sits in a stream, where it could hold back later launches that
    // share its hardware queue)
    std::vector<cudaEvent_t> ev_pool;

    Batch batch;
    size_t budget = 0, used = 0;
    int max_streams = 0;
    int admitting = 0;                     // sessions between the queue and the batch
    int max_inflight = 3, max_pending = 8;
    std::mutex mu;
    std::condition_variable cv;
    std::thread th, th_alloc;
    std::deque<int> to_make;               // admitted, state not yet allocated
    std::deque<std::pair<int, Session*>> made;   // allocated (null: failed), not yet inserted
    std::condition_variable cv_alloc;
    bool stop = false;
    bool hold = false;                     // no new ticks while set (frames collect)
    std::string err;                       // first dispatcher failure (sticky)
    std::vector<Sess> sess;
    std::deque<int> queue;                 // sessions waiting for admission
    std::deque<Tick*> inflight;
    std::vector<float> lat_ms, wait_ms;
    long long ticks = 0, frames_done = 0, admitted = 0;
    double mpix_done = 0, t_stats = 0;
    double host_sum = 0, host_max = 0, span_sum = 0, span_max = 0, admit_max = 0, retire_max = 0;
    long long spans = 0;

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        cv_alloc.notify_all();
        if (th.joinable()) th.join();
        if (th_alloc.joinable()) th_alloc.join();
        batch.sync();
        for (Tick* t : inflight) {
            if (t->ev) cudaEventDestroy(t->ev);
            delete t;
        }
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        for (auto& m : made) delete m.second;
    }

    bool init(int device, size_t budget_bytes, int max_n) {
        budget = budget_bytes;
        max_streams = max_n;
        if (!batch.init(device, max_n)) return false;
        if (!reserve()) return false;
        t_stats = now_ms();
        th = std::thread([this] { run(); });
        th_alloc = std::thread([this] { run_alloc(); });
        return true;
    }

    // The budget (at most the device's free memory less 2 GiB) is reserved in
    // the device's stream-ordered pool before serving starts: one allocation,
    // freed back to the pool, which keeps it (its release threshold is
    // raised).  Sessions' state is then carved from reserved memory, so an
    // admission does not grow the pool - growing it maps new physical memory,
    // which blocked the dispatcher's launches for tens of milliseconds.
    bool reserve() {
        size_t free_b = 0, total_b = 0;
        if (!cuda_ok(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo")) return false;
        const size_t margin = (size_t)2 << 30;
        const size_t want = std::min(budget, free_b > margin ? free_b - margin : (size_t)0);
        if (want == 0) return true;
        void* p = nullptr;
        if (!cuda_ok(cudaMallocAsync(&p, want, batch.st_alloc), "cudaMallocAsync(reserve)")) return false;
        if (!cuda_ok(cudaFreeAsync(p, batch.st_alloc), "cudaFreeAsync(reserve)")) return false;
        return cuda_ok(cudaStreamSynchronize(batch.st_alloc), "reserve sync");
    }

    // allocation thread: Batch::make touches no batch state
    void run_alloc() {
        cudaSetDevice(batch.device);
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            cv_alloc.wait(lk, [&] { return stop || !to_make.empty(); });
            if (stop) return;
            const int i = to_make.front();
            to_make.pop_front();
            const wema_cuda_config cfg = sess[i].cfg;
            lk.unlock();
            const double t0 = now_ms();
            Session* s = batch.make(cfg);
            if (!s) {                  // the pool may hold reserved memory it cannot split: release it, retry
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, batch.device) == cudaSuccess &&
                    cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
                    s = batch.make(cfg);
            }
            const double dt = now_ms() - t0;
            const std::string why = s ? "" : last_error();
            lk.lock();
            admit_max = std::max(admit_max, dt);
            if (!s) sess[i].err = why;
            made.push_back({i, s});
            cv.notify_all();
        }
    }

    cudaEvent_t take_event() {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        return cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate") ? e : nullptr;
    }

    int live() const {
        int n = 0;
        for (const Sess& s : sess) n += s.state == WEMA_CUDA_SESSION_LIVE;
        return n;
    }

    // ---- dispatcher (all Batch calls happen on this thread)
    void fail(const char* what) {
        if (err.empty()) err = std::string(what) + ": " + last_error();
    }

    void reap() {
        bool any = false;
        while (!inflight.empty()) {
            Tick* t = inflight.front();
            if (t->t_done < 0) {
                const cudaError_t q = cudaEventQuery(t->ev);
                if (q == cudaErrorNotReady) break;
                t->t_done = now_ms();
                if (q != cudaSuccess && err.empty()) err = std::string("tick: ") + cudaGetErrorString(q);
            }
            inflight.pop_front();
            any = true;
            const double span = t->t_done - t->t_issue;
            span_sum += span;
            span_max = std::max(span_max, span);
            spans++;
            for (size_t k = 0; k < t->sids.size(); k++) {
                Sess& s = sess[t->sids[k]];
                s.completed++;
                s.inflight--;
                frames_done++;
                mpix_done += (double)s.cfg.width * s.cfg.height * 1e-6;
                lat_ms.push_back((float)(t->t_done - t->t_submit[k]));
            }
            ev_pool.push_back(t->ev);
            delete t;
        }
        if (any) cv.notify_all();   // drain() and submitters wait on progress
    }

    // (sess may grow while the lock is released: entries are re-indexed after)
    void retire(std::unique_lock<std::mutex>& lk) {
        for (size_t i = 0; i < sess.size(); i++) {
            const Sess& s = sess[i];
            if (s.state != WEMA_CUDA_SESSION_LIVE || !s.closing || !s.pending.empty() || s.inflight) continue;
            const int bid = s.bid;
            lk.unlock();
            const double t0 = now_ms();
            const bool ok = batch.remove(bid, false);   // its last tick has completed
            const double dt = now_ms() - t0;
            lk.lock();
            retire_max = std::max(retire_max, dt);
            if (!ok) fail("close");
            Sess& t = sess[i];
            t.state = WEMA_CUDA_SESSION_CLOSED;
            t.bid = -1;
            used -= t.bytes;
        }
    }

    // the queue's head goes to the allocation thread while its state fits
    // the budget; allocated sessions join the batch here
    void admit() {
        while (!queue.empty()) {
            const int i = queue.front();
            if (used + sess[i].bytes > budget || live() + admitting >= max_streams) break;
            queue.pop_front();
            used += sess[i].bytes;
            admitting++;
            to_make.push_back(i);
            cv_alloc.notify_one();
        }
        while (!made.empty()) {
            const int i = made.front().first;
            Session* s = made.front().second;
            made.pop_front();
            admitting--;
            Sess& t = sess[i];
            const int bid = s ? batch.insert(s) : -1;
            if (bid < 0) {                      // e.g. the device ran out of memory
                if (t.err.empty()) t.err = last_error();
                used -= t.bytes;
                t.state = WEMA_CUDA_SESSION_FAILED;
                continue;
            }
            t.bid = bid;
            t.state = WEMA_CUDA_SESSION_LIVE;
            t.t_admit = now_ms();
            wait_ms.push_back((float)(t.t_admit - t.t_open));
            admitted++;
        }
    }

    bool idle() const {
        if (!inflight.empty() || !queue.empty() || admitting) return false;
        for (const Sess& s : sess)
            if (s.state == WEMA_CUDA_SESSION_LIVE && !s.pending.empty()) return false;
        return true;
    }

    void run() {
        cudaSetDevice(batch.device);
        std::unique_lock<std::mutex> lk(mu);
        std::vector<int> ids;
        std::vector<const uint8_t*> in;
        std::vector<uint8_t*> out;
        while (true) {
            reap();
            retire(lk);
            admit();
            if (stop && inflight.empty()) break;
            if ((int)inflight.size() < max_inflight && err.empty() && !hold) {
                Tick* t = new Tick();
                t->srv = this;
                t->ev = take_event();
                if (!t->ev) {
                    fail("tick event");
                    delete t;
                    continue;
                }
                ids.clear();
                in.clear();
                out.clear();
                for (size_t i = 0; i < sess.size(); i++) {
                    Sess& s = sess[i];
                    if (s.state != WEMA_CUDA_SESSION_LIVE || s.pending.empty()) continue;
                    const Frame f = s.pending.front();
                    s.pending.pop_front();
                    s.inflight++;
                    ids.push_back(s.bid);
                    in.push_back(f.in);
                    out.push_back(f.out);
                    t->sids.push_back((int)i);
                    t->t_submit.push_back(f.t_submit);
                }
                if (!ids.empty()) {
                    inflight.push_back(t);
                    ticks++;
                    t->t_issue = now_ms();
                    lk.unlock();
                    bool ok = batch.tick(ids.data(), in.data(), out.data(), (int)ids.size(), nullptr, t->ev);
                    const std::string why = ok ? "" : last_error();
                    const double dt = now_ms() - t->t_issue;
                    lk.lock();
                    host_sum += dt;
                    host_max = std::max(host_max, dt);
                    if (!ok) {
                        if (err.empty()) err = "tick: " + why;
                        t->t_done = now_ms();           // nothing of it will complete later
                    }
                    continue;
                }
                ev_pool.push_back(t->ev);
                delete t;
            }
            // ticks in flight: poll their events often; else wait for work
            if (inflight.empty()) cv.wait_for(lk, std::chrono::milliseconds(2));
            else cv.wait_for(lk, std::chrono::microseconds(50));
        }
    }

    // ---- client side
    int open(const wema_cuda_config& c) {
        const size_t bytes = Session::bytes_for(c, 1);
        if (bytes == 0) return -1;                 // invalid config (error set)
        if (!c.use_iir) { set_error("served streams use the IIR filter (use_iir = 1)"); return -1; }
        if (c.device != batch.device) { set_error("stream device %d differs from the server's %d", c.device, batch.device); return -1; }
        std::lock_guard<std::mutex> lk(mu);
        if (bytes > budget) {
            set_error("stream state (%zu bytes) exceeds the whole budget (%zu bytes)", bytes, budget);
            return -1;
        }
        Sess s;
        s.cfg = c;
        s.bytes = bytes;
        s.t_open = now_ms();
        sess.push_back(s);
        const int id = (int)sess.size() - 1;
        queue.push_back(id);
        cv.notify_all();
        return id;
    }
};

}  // namespace wema

// ===================================================================== C ABI
using namespace wema;

struct wema_cuda_server {
    Server s;
};

#define WEMA_API extern "C" __attribute__((visibility("default")))

static bool server_sess(wema_cuda_server* v, int sid) {
    if (sid < 0 || sid >= (int)v->s.sess.size()) {
        set_error("no session %d", sid);
        return false;
    }
    return true;
}

WEMA_API int wema_cuda_server_create(int device, size_t budget_bytes, int max_streams, wema_cuda_server** out) {
    clear_error();
    if (!out || max_streams < 1 || budget_bytes == 0) { set_error("bad argument"); return -1; }
    *out = nullptr;
    wema_cuda_server* v = new (std::nothrow) wema_cuda_server();
    if (!v) { set_error("out of host memory"); return -1; }
    if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice") || !v->s.init(device, budget_bytes, max_streams)) {
        delete v;
        return -1;
    }
    *out = v;
    return 0;
}

WEMA_API void wema_cuda_server_destroy(wema_cuda_server* v) {
    if (!v) return;
    cudaSetDevice(v->s.batch.device);
    delete v;
}

WEMA_API int wema_cuda_server_open(wema_cuda_server* v, const wema_cuda_config* cfg, int* sid) {
    clear_error();
    if (!v || !cfg || !sid) { set_error("null argument"); return -1; }
    const int id = v->s.open(*cfg);
    if (id < 0) return -1;
    *sid = id;
    return 0;
}

WEMA_API int wema_cuda_server_submit(wema_cuda_server* v, int sid, const void* d_in_u8, void* d_out_u8) {
    clear_error();
    if (!v || !d_in_u8 || !d_out_u8) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(v->s.mu);
    if (!v->s.err.empty()) { set_error("%s", v->s.err.c_str()); return -1; }
    if (!server_sess(v, sid)) return -1;
    Server::Sess& s = v->s.sess[sid];
    if (s.state == WEMA_CUDA_SESSION_QUEUED) {
        s.dropped++;
        return 1;
    }
    if (s.state != WEMA_CUDA_SESSION_LIVE || s.closing) { set_error("session %d is closed", sid); return -1; }
    if ((int)s.pending.size() >= v->s.max_pending) {
        s.dropped++;
        return 2;
    }
    s.pending.push_back({(const uint8_t*)d_in_u8, (uint8_t*)d_out_u8, now_ms()});
    s.submitted++;
    v->s.cv.notify_all();
    return 0;
}

WEMA_API int wema_cuda_server_close(wema_cuda_server* v, int sid) {
    clear_error();
    if (!v) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(v->s.mu);
    if (!server_sess(v, sid)) return -1;
    Server::Sess& s = v->s.sess[sid];
    if (s.state == WEMA_CUDA_SESSION_QUEUED) {
        // (absent when the dispatcher is admitting it right now: it then
        // becomes live with `closing` set and is retired at once)
        auto it = std::find(v->s.queue.begin(), v->s.queue.end(), sid);
        if (it != v->s.queue.end()) {
            v->s.queue.erase(it);
            s.state = WEMA_CUDA_SESSION_CLOSED;
        }
    }
    s.closing = true;
    v->s.cv.notify_all();
    return 0;
}

WEMA_API int wema_cuda_server_poll(wema_cuda_server* v, int sid, wema_cuda_session_status* st) {
    clear_error();
    if (!v || !st) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(v->s.mu);
    if (!server_sess(v, sid)) return -1;
    const Server::Sess& s = v->s.sess[sid];
    st->state = s.state;
    st->submitted = s.submitted;
    st->completed = s.completed;
    st->dropped = s.dropped;
    st->state_bytes = s.bytes;
    st->admission_wait_ms = s.state == WEMA_CUDA_SESSION_QUEUED ? -1.0 : s.t_admit - s.t_open;
    if (s.state == WEMA_CUDA_SESSION_FAILED) set_error("%s", s.err.c_str());
    return 0;
}

WEMA_API int wema_cuda_server_hold(wema_cuda_server* v, int hold) {
    clear_error();
    if (!v) { set_error("null argument"); return -1; }
    {
        std::lock_guard<std::mutex> lk(v->s.mu);
        v->s.hold = hold != 0;
    }
    v->s.cv.notify_all();
    return 0;
}

WEMA_API int wema_cuda_server_drain(wema_cuda_server* v, int timeout_ms) {
    clear_error();
    if (!v) { set_error("null argument"); return -1; }
    std::unique_lock<std::mutex> lk(v->s.mu);
    if (v->s.hold) { set_error("drain: the server is held"); return -1; }
    const bool ok = v->s.cv.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                     [&] { return !v->s.err.empty() || v->s.idle(); });
    if (!v->s.err.empty()) { set_error("%s", v->s.err.c_str()); return -1; }
    if (!ok) { set_error("drain: frames still pending after %d ms", timeout_ms); return -1; }
    return 0;
}

WEMA_API int wema_cuda_server_stats(wema_cuda_server* v, int reset, wema_cuda_serve_stats* out) {
    clear_error();
    if (!v || !out) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(v->s.mu);
    Server& s = v->s;
    const double t = now_ms();
    out->seconds = (t - s.t_stats) * 1e-3;
    out->ticks = s.ticks;
    out->frames = s.frames_done;
    out->mpix_frames = s.mpix_done;
    out->latency_p50_ms = pct(s.lat_ms, 0.50);
    out->latency_p99_ms = pct(s.lat_ms, 0.99);
    out->latency_max_ms = s.lat_ms.empty() ? 0.f : *std::max_element(s.lat_ms.begin(), s.lat_ms.end());
    out->admission_wait_p50_ms = pct(s.wait_ms, 0.50);
    out->admission_wait_max_ms = s.wait_ms.empty() ? 0.f : *std::max_element(s.wait_ms.begin(), s.wait_ms.end());
    out->sessions_admitted = s.admitted;
    out->sessions_live = s.live();
    out->sessions_queued = (int)s.queue.size();
    out->bytes_used = s.used;
    out->budget_bytes = s.budget;
    out->launches = s.batch.launches;
    out->tick_host_ms_mean = s.ticks ? (float)(s.host_sum / s.ticks) : 0.f;
    out->tick_host_ms_max = (float)s.host_max;
    out->tick_span_ms_mean = s.spans ? (float)(s.span_sum / s.spans) : 0.f;
    out->tick_span_ms_max = (float)s.span_max;
    out->admit_ms_max = (float)s.admit_max;
    out->retire_ms_max = (float)s.retire_max;
    if (reset) {
        s.host_sum = s.host_max = s.span_sum = s.span_max = s.admit_max = s.retire_max = 0;
        s.spans = 0;
        s.lat_ms.clear();
        s.wait_ms.clear();
        s.ticks = 0;
        s.frames_done = 0;
        s.mpix_done = 0;
        s.admitted = 0;
        s.t_stats = t;
    }
    return s.err.empty() ? 0 : (set_error("%s", s.err.c_str()), -1);
}
