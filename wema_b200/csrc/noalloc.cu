// noalloc.cu - the exact threshold without any device allocation.
//
// Some callers cannot allocate device memory once they are running: a host
// application that owns every byte of the GPU through its own pool, a
// real-time loop where cudaMalloc's implicit device synchronisation would
// stall the frame, or a plugin that may only use buffers its host hands it.
// For them wema_cuda_threshold_flat_noalloc does what wema_cuda_threshold_flat
// does with its scratch in a fixed array compiled into this library instead
// of a cudaMallocAsync'd block.  The caller still passes the input array and
// the output scalars.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it (kNoAllocScratchBytes) until the process exits, and every
// call on that GPU shares it.  Host code cannot use the variable's name as a
// device address, so the first call on each device (with that device current)
// looks the address up with cudaGetSymbolAddress and caches it.
#include <mutex>

#include "session.h"
#include "wema_cuda.h"

namespace wema {

// Largest input: 2^24 floats, more than a 3840x2160 frame's 6-slot
// coefficient array (16,524,000).  Its threshold scratch needs 2,883,840 bytes.
constexpr size_t kNoAllocMaxElems = (size_t)1 << 24;
constexpr size_t kNoAllocScratchBytes = (size_t)1 << 22;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};
}  // namespace

// device address of g_noalloc_scratch on the current device (looked up once)
static void* noalloc_scratch(int dev) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error("cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            return nullptr;
        }
        g_noalloc_addr[dev] = p;
    }
    return g_noalloc_addr[dev];
}

}  // namespace wema

using namespace wema;

extern "C" __attribute__((visibility("default"))) int wema_cuda_threshold_flat_noalloc(
    const float* d_x, size_t n, int threshold_form, float* d_thr, float* d_sum, void* cuda_stream) {
    clear_error();
    if (!d_x || !d_thr || n == 0) {
        set_error("bad argument: need an input array, n > 0 and a threshold output");
        return -1;
    }
    if (n > kNoAllocMaxElems) {
        set_error("n = %zu exceeds the allocation-free maximum of %zu elements", n,
                  kNoAllocMaxElems);
        return -1;
    }
    const size_t need = thr_scratch_bytes((long long)n);
    if (need > kNoAllocScratchBytes) {   // cannot happen for n <= kNoAllocMaxElems
        set_error("scratch of %zu bytes exceeds the static %zu", need, kNoAllocScratchBytes);
        return -1;
    }
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return -1;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device %d out of range", dev);
        return -1;
    }
    void* scratch = noalloc_scratch(dev);
    if (!scratch) return -1;
    // Nothing in the scratch has to start at zero: the kernels write every
    // partial sum, prefix and candidate entry before reading it, the first
    // kernel clears the lane counter, and the binade history (which a
    // previous call may have left) is not consulted.
    ThrScratch ts{};
    thr_scratch_bind(ts, scratch, (long long)n);
    PyrView v{};
    v.coef = d_x;
    v.levels = 0;
    v.off6[0] = (long long)n;
    return cuda_ok(launch_threshold(&v, 1, &ts, d_thr, d_sum, threshold_form, 0, 0,
                                    (cudaStream_t)cuda_stream),
                   "threshold")
               ? 0
               : -1;
}
