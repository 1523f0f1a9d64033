// gtc_static.cu -- a counting entry point that allocates no device memory.
//
// Some callers cannot allocate device memory at the moment they count: a
// request loop that reserved all of its memory at start-up and must not grow
// afterwards, a plug-in living inside a framework whose caching allocator owns
// the device memory, or a caller that cannot afford the implicit device-wide
// synchronisation a cudaMalloc/cudaFree may cause.  gtc_count_noalloc serves
// them: the caller still passes the graph and the output buffers, but the
// counting pipeline's scratch space (forward lists, per-vertex records, work
// queues, accumulators) lives in one fixed array compiled into this library.
//
// Limits and rules:
//   * the array holds kStaticScratchBytes (32 MiB); a graph whose workspace
//     (gtc_workspace_size) is larger is rejected with GTC_ERR_CAPACITY before
//     any device work -- about 48 bytes per vertex plus 4.5 bytes per
//     adjacency entry plus 67 KiB, e.g. 100,000 vertices with 4 million
//     entries fit;
//   * every device that loads the library holds the array until the process
//     exits;
//   * the array is shared by all calls on a device and keeps the last call's
//     contents; each call clears what must start at zero itself, but two calls
//     whose work overlaps on the GPU (different streams, no ordering between
//     them) race on it and must be serialised by the caller;
//   * the first call on each device looks the array's device address up
//     (cudaGetSymbolAddress); make that first call before any stream capture.
//     The address is kept for the life of the process; a cudaDeviceReset
//     makes it stale, so a process that resets a device must not use this
//     entry point on that device afterwards.
// The entry point calls no cudaMalloc, cudaFree or other allocating routine.
#include <mutex>

#include "gtc_core.cuh"

namespace gtc {
namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;

// The scratch array.  In host code this name is only a host-side stand-in for
// the device object, never a device address: host code must use the address
// returned by cudaGetSymbolAddress for the current device.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void *g_static_addr[64];   // per device, set once

// Device address of g_static_scratch on the current device (looked up on the
// first call per device, with that device current).
gtc_status static_scratch(void **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GTC_ERR_CUDA;
    if (dev < 0 || dev >= 64) return GTC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p)
            return GTC_ERR_CUDA;
        g_static_addr[dev] = p;
    }
    *out = g_static_addr[dev];
    return GTC_OK;
}

}  // namespace
}  // namespace gtc

using namespace gtc;

extern "C" gtc_status gtc_count_noalloc(const void *d_off, int off_bits, const int32_t *d_ind,
                                        int64_t n, int64_t nnz, gtc_mode mode, int64_t *d_r,
                                        int64_t *d_t, double *d_lcc, int64_t *d_global,
                                        gtc_stream_t stream)
{
    size_t need = 0;
    gtc_status st = gtc_workspace_size(n, nnz, off_bits, mode, &need);
    if (st != GTC_OK) return st;
    if (need > kStaticScratchBytes) return GTC_ERR_CAPACITY;
    if (!d_off || (nnz > 0 && !d_ind)) return GTC_ERR_INVALID_ARGUMENT;
    if (mode == GTC_MODE_ORIENTED && (d_r || d_t || d_lcc)) return GTC_ERR_INVALID_ARGUMENT;
    void *ws = nullptr;
    st = static_scratch(&ws);
    if (st != GTC_OK) return st;
    const bool pv = mode == GTC_MODE_PLAIN;
    const RowConfig cfg = pick_row_config(n, nnz);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    long long *r = reinterpret_cast<long long *>(d_r);
    long long *t = reinterpret_cast<long long *>(d_t);
    long long *g = reinterpret_cast<long long *>(d_global);
    if (off_bits == 32)
        return run_count<int>(static_cast<const int *>(d_off), d_ind, n, nnz, pv, r, t, d_lcc, g,
                              ws, kStaticScratchBytes, s, cfg, nullptr);
    return run_count<long long>(static_cast<const long long *>(d_off), d_ind, n, nnz, pv, r, t,
                                d_lcc, g, ws, kStaticScratchBytes, s, cfg, nullptr);
}
