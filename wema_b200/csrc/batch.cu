// batch.cu - C ABI of the batched streams (wema_cuda_batch_*); the Batch
// class itself is in batch.h.
#include <mutex>
#include <new>

#include "batch.h"

namespace wema {

__global__ void k_table_copy(uint4* __restrict__ dst, const uint4* __restrict__ src, size_t n16) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

cudaError_t launch_table_copy(void* dst, const void* host_mapped, size_t bytes, cudaStream_t st) {
    const size_t n16 = (bytes + 15) / 16;
    if (n16 == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<size_t>((n16 + 255) / 256, 148);
    k_table_copy<<<blocks, 256, 0, st>>>(static_cast<uint4*>(dst), static_cast<const uint4*>(host_mapped), n16);
    return cudaGetLastError();
}

}  // namespace wema

// ===================================================================== C ABI
using namespace wema;

struct wema_cuda_batch {
    Batch b;
    std::mutex mu;
};

#define WEMA_API extern "C" __attribute__((visibility("default")))

WEMA_API size_t wema_cuda_batch_stream_bytes(const wema_cuda_config* cfg) {
    clear_error();
    if (!cfg) { set_error("null config"); return 0; }
    return Session::bytes_for(*cfg, 1);
}

WEMA_API int wema_cuda_batch_create(int device, int max_streams, wema_cuda_batch** out) {
    clear_error();
    if (!out || max_streams < 1) { set_error("bad argument"); return -1; }
    *out = nullptr;
    wema_cuda_batch* b = new (std::nothrow) wema_cuda_batch();
    if (!b) { set_error("out of host memory"); return -1; }
    if (!b->b.init(device, max_streams)) {
        delete b;
        return -1;
    }
    *out = b;
    return 0;
}

WEMA_API void wema_cuda_batch_destroy(wema_cuda_batch* b) {
    if (!b) return;
    cudaSetDevice(b->b.device);
    delete b;
}

WEMA_API int wema_cuda_batch_add(wema_cuda_batch* b, const wema_cuda_config* cfg, int* id) {
    clear_error();
    if (!b || !cfg || !id) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    const int k = b->b.add(*cfg);
    if (k < 0) return -1;
    *id = k;
    return 0;
}

WEMA_API int wema_cuda_batch_remove(wema_cuda_batch* b, int id) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    return b->b.remove(id) ? 0 : -1;
}

WEMA_API int wema_cuda_batch_tick(wema_cuda_batch* b, const int* ids, const void* const* d_in_u8,
                                  void* const* d_out_u8, int n, void* wait_event, void* done_event) {
    clear_error();
    if (!b || n < 0 || (n > 0 && (!ids || !d_in_u8 || !d_out_u8))) { set_error("bad argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    if (n == 0) {
        if (done_event && !cuda_ok(cudaEventRecord((cudaEvent_t)done_event, b->b.st_xfer), "event record"))
            return -1;
        return 0;
    }
    return b->b.tick(ids, (const uint8_t* const*)d_in_u8, (uint8_t* const*)d_out_u8, n,
                     (cudaEvent_t)wait_event, (cudaEvent_t)done_event)
               ? 0
               : -1;
}

WEMA_API int wema_cuda_batch_tick_host(wema_cuda_batch* b, const int* ids, const void* const* h_in_u8,
                                       void* const* h_out_u8, int n, void* wait_event, void* done_event) {
    clear_error();
    if (!b || n < 1 || !ids || !h_in_u8 || !h_out_u8) { set_error("bad argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    return b->b.tick_host(ids, (const uint8_t* const*)h_in_u8, (uint8_t* const*)h_out_u8, n,
                          (cudaEvent_t)wait_event, (cudaEvent_t)done_event)
               ? 0
               : -1;
}

WEMA_API int wema_cuda_batch_set_graphs(wema_cuda_batch* b, int enable) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    b->b.use_graphs = enable != 0;
    return 0;
}

WEMA_API int wema_cuda_batch_set_groups(wema_cuda_batch* b, int groups) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    if (groups < 1 || groups > wema::Batch::MAXG) {
        set_error("groups %d outside 1..%d", groups, wema::Batch::MAXG);
        return -1;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    b->b.groups = groups;
    return 0;
}

WEMA_API int wema_cuda_batch_set_host_overlap(wema_cuda_batch* b, int enable) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    b->b.host_overlap = enable != 0;
    return 0;
}

WEMA_API int wema_cuda_batch_set_timing(wema_cuda_batch* b, int enable) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    if (!b->b.sync()) return -1;
    for (auto& t : b->b.tb)
        if (!b->b.collect(t)) return -1;
    b->b.timing = enable != 0;
    return 0;
}

WEMA_API int wema_cuda_batch_stage_times(wema_cuda_batch* b, double* times_ms, long long* ticks) {
    clear_error();
    if (!b || !times_ms || !ticks) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    return b->b.stage_times(times_ms, ticks) ? 0 : -1;
}

WEMA_API size_t wema_cuda_batch_snapshot_bytes(wema_cuda_batch* b, int id) {
    clear_error();
    if (!b) { set_error("null argument"); return 0; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= (int)b->b.streams.size() || !b->b.streams[id]) { set_error("no stream %d", id); return 0; }
    return b->b.streams[id]->snapshot_bytes();
}

WEMA_API int wema_cuda_batch_snapshot(wema_cuda_batch* b, int id, void* host, size_t cap) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= (int)b->b.streams.size() || !b->b.streams[id]) { set_error("no stream %d", id); return -1; }
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice") || !b->b.sync()) return -1;
    return b->b.streams[id]->snapshot(host, cap) ? 0 : -1;
}

WEMA_API int wema_cuda_batch_restore(wema_cuda_batch* b, int id, const void* host, size_t bytes) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= (int)b->b.streams.size() || !b->b.streams[id]) { set_error("no stream %d", id); return -1; }
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice") || !b->b.sync()) return -1;
    return b->b.streams[id]->restore(host, bytes) ? 0 : -1;
}

WEMA_API int wema_cuda_batch_sync(wema_cuda_batch* b) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (!cuda_ok(cudaSetDevice(b->b.device), "cudaSetDevice")) return -1;
    return b->b.sync() ? 0 : -1;
}

WEMA_API int wema_cuda_batch_stats(wema_cuda_batch* b, long long* ticks, long long* launches, int* live) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (ticks) *ticks = b->b.ticks;
    if (launches) *launches = b->b.launches;
    if (live) *live = b->b.live();
    return 0;
}

WEMA_API int wema_cuda_batch_read(wema_cuda_batch* b, int id, int what, int channel, void* host,
                                  size_t bytes) {
    clear_error();
    if (!b) { set_error("null argument"); return -1; }
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= (int)b->b.streams.size() || !b->b.streams[id]) { set_error("no stream %d", id); return -1; }
    if (!b->b.sync()) return -1;
    if (what != WEMA_CUDA_READ_THRESHOLD) { set_error("batched streams expose the threshold only"); return -1; }
    Session& S = *b->b.streams[id];
    if (channel < 0 || channel >= S.nch || bytes < sizeof(float)) { set_error("bad channel or size"); return -1; }
    return cuda_ok(cudaMemcpy(host, S.slot[0].thr + channel, sizeof(float), cudaMemcpyDeviceToHost), "read")
               ? (int)sizeof(float)
               : -1;
}
