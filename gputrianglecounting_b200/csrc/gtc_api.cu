// gtc_api.cu -- the C ABI (include/gtc_b200.h): status strings, workspace
// sizing, the counting entry points, the CSR validator, the vertex-subset
// kernel and the reference-compatible kernelCall shims.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "gtc_core.cuh"

namespace cg = cooperative_groups;

namespace gtc {
namespace {

inline cudaStream_t as_stream(gtc_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// ================================================================ validator

// The reason word starts at kNoReason (every byte 0x7f) so that atomicMin
// keeps the smallest failing reason code; it maps back to GTC_CSR_OK.
constexpr int kNoReason = 0x7f7f7f7f;

// Phase 1: offsets start at 0, end at nnz, never decrease.
template <typename OffT>
__global__ void validate_offsets_kernel(const OffT *__restrict__ off, long long n,
                                        long long nnz, int *reason)
{
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v == 0 && ((long long)off[0] != 0 || (long long)off[n] != nnz))
        atomicMin(reason, GTC_CSR_BAD_OFFSETS);
    if (v < n && (long long)off[v + 1] < (long long)off[v])
        atomicMin(reason, GTC_CSR_BAD_OFFSETS);
}

// Phase 2 (warp per row): ids in range, no self-loop, strictly ascending.
template <typename OffT>
__global__ void validate_rows_kernel(const OffT *__restrict__ off,
                                     const int *__restrict__ ind, long long n,
                                     int *reason)
{
    if (*(volatile int *)reason != kNoReason) return;
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long a = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < n; a += warps) {
        const long long rb = off[a], re = off[a + 1];
        int bad = GTC_CSR_OK + 100;
        for (long long e = rb + lane; e < re; e += 32) {
            const int x = ind[e];
            if ((unsigned long long)(long long)x >= (unsigned long long)n) bad = min(bad, (int)GTC_CSR_INDEX_RANGE);
            else if (x == a) bad = min(bad, (int)GTC_CSR_SELF_LOOP);
            if (e > rb && ind[e - 1] >= x) bad = min(bad, (int)GTC_CSR_UNSORTED_OR_DUPLICATE);
        }
        if (bad != GTC_CSR_OK + 100) atomicMin(reason, bad);
    }
}

// Phase 3: every (a, x) has its mirror (x, a).  Warps take 32-entry strides
// of the adjacency (so a hub row is spread over many warps); each lane finds
// its entry's row from the stride's first row.
template <typename OffT>
__global__ void validate_symmetry_kernel(const OffT *__restrict__ off,
                                         const int *__restrict__ ind, long long n,
                                         long long nnz, int *reason,
                                         unsigned long long *counts)
{
    // Rows are strictly ascending without self-loops (checked before), so
    // reversal maps the entries (a, x) with a < x injectively onto those with
    // a > x: the graph is symmetric iff every such upper entry's reverse is
    // present and both kinds are equally many (counts[0] vs counts[1]).  Only
    // upper entries are searched for, half of all entries.
    if (*(volatile int *)reason != kNoReason) return;
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long upper = 0, lower = 0;
    bool ok = true;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 < nnz;
         w += warps) {
        const long long e = w * 32 + lane;
        long long a = 0;
        if (lane == 0) a = row_of_entry(off, n, w * 32);
        a = __shfl_sync(0xffffffffu, a, 0);
        if (e < nnz) {
            while ((long long)off[a + 1] <= e) ++a;
            const int x = ind[e];
            if (x < a) {
                ++lower;
            } else {
                ++upper;
                long long lo = off[x], hi = off[x + 1];
                while (lo < hi) {
                    const long long mid = (lo + hi) >> 1;
                    if (ind[mid] < a) lo = mid + 1; else hi = mid;
                }
                if (lo >= (long long)off[x + 1] || ind[lo] != a) ok = false;
            }
        }
    }
    if (!__all_sync(0xffffffffu, ok) && lane == 0) atomicMin(reason, GTC_CSR_ASYMMETRIC);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        upper += __shfl_down_sync(0xffffffffu, upper, d);
        lower += __shfl_down_sync(0xffffffffu, lower, d);
    }
    if (lane == 0) {
        if (upper) atomicAdd(&counts[0], upper);
        if (lower) atomicAdd(&counts[1], lower);
    }
}

template <typename OffT>
gtc_status run_validate(const OffT *off, const int *ind, long long n, long long nnz,
                        void *ws, int32_t *h_reason, cudaStream_t stream)
{
    int *reason = static_cast<int *>(ws);
    unsigned long long *counts =
        reinterpret_cast<unsigned long long *>(static_cast<char *>(ws) + 64);
    cudaError_t e = cudaMemsetAsync(reason, 0x7f, sizeof(int), stream);
    if (e != cudaSuccess) return GTC_ERR_CUDA;
    e = cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return GTC_ERR_CUDA;
    const unsigned vb = (unsigned)div_up<long long>(n + 1, 256);
    validate_offsets_kernel<<<vb, 256, 0, stream>>>(off, n, nnz, reason);
    if (n > 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        long long want = div_up<long long>(n, 8);
        unsigned blocks = (unsigned)(want < (long long)sms * 16 ? want : (long long)sms * 16);
        validate_rows_kernel<<<blocks, 256, 0, stream>>>(off, ind, n, reason);
        if (nnz > 0) {
            const long long swant = div_up<long long>(nnz, 32 * 8);
            const unsigned sblocks =
                (unsigned)(swant < (long long)sms * 16 ? swant : (long long)sms * 16);
            validate_symmetry_kernel<<<sblocks, 256, 0, stream>>>(off, ind, n, nnz, reason,
                                                                  counts);
        }
    }
    // reason word and the two entry counts in one read
    unsigned char host[80];
    e = cudaMemcpyAsync(host, ws, sizeof(host), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return GTC_ERR_CUDA;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return GTC_ERR_CUDA;
    int r = 0;
    unsigned long long c[2] = {0, 0};
    std::memcpy(&r, host, sizeof(int));
    std::memcpy(c, host + 64, sizeof(c));
    if (r == kNoReason && c[0] != c[1]) r = GTC_CSR_ASYMMETRIC;
    *h_reason = r == kNoReason ? GTC_CSR_OK : r;
    return GTC_OK;
}

// ============================================================ vertex subset

constexpr int kSubThreads = 256;
constexpr int kSubSlots = 4096;
constexpr long long kSubHubMin = kSubSlots / 2;   // longer listed rows go to the hub kernel
constexpr int kSubHubThreads = 1024;
constexpr long long kSubHubBits = 1ll << 20;      // bitmap span of a hub row (128 KiB)

template <typename IndT>
__device__ __forceinline__ bool sorted_contains(const IndT *__restrict__ list,
                                                long long len, long long key)
{
    long long lo = 0, hi = len;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if ((long long)list[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo < len && (long long)list[lo] == key;
}

// |N(u) ∩ N(v)| by binary search of the shorter sorted row in the longer,
// this lane's share (lane stride 32).
template <typename IndT>
__device__ __forceinline__ unsigned long long search_shorter(const IndT *__restrict__ ind,
                                                             long long vb, long long dv,
                                                             long long ub, long long du,
                                                             int lane)
{
    unsigned long long acc = 0;
    if (du < dv) {
        for (long long i = lane; i < du; i += 32)
            acc += sorted_contains(ind + vb, dv, (long long)ind[ub + i]);
    } else {
        for (long long i = lane; i < dv; i += 32)
            acc += sorted_contains(ind + ub, du, (long long)ind[vb + i]);
    }
    return acc;
}

__device__ __forceinline__ void add_out(long long *o, unsigned long long x)
{
    atomicAdd(reinterpret_cast<unsigned long long *>(o), x);
}
__device__ __forceinline__ void add_out(int *o, unsigned long long x)
{
    atomicAdd(o, (int)x);
}

// out[k] = sum over u in N(v) of |N(v) ∩ N(u)|, v = vertex[k], with full
// adjacency lists (the rows of the listed vertices and of their neighbours
// are the only ones read, as in the reference's vertex-list kernel,
// src/clusteringCount.cu:266-312).  Edges with u == v or a list shorter
// than two are skipped like the reference (:292-294).  Two kernels:
//   * subset_kernel, a block per listed vertex of degree <= kSubHubMin: N(v)
//     goes to a shared hash table; for each neighbour u, N(u) is probed into
//     the table when it is not much longer, otherwise the shorter row is
//     binary-searched in the longer.  It writes 0 for the longer rows;
//   * subset_hub_kernel, all blocks on every longer ("hub") row: each block
//     sets N(v) in a shared bitmap over the row's id span and takes every
//     gridDim.x-th neighbour, whose row its warps probe into the bitmap with
//     coalesced loads; neighbour rows longer than 2,048 entries are queued
//     and swept afterwards by all of the block's warps in 1,024-entry pieces,
//     so that no warp is left alone with a hub's row; block sums are added to
//     out[k].  A row whose span exceeds the bitmap falls back to the binary
//     search.
// Spreading a hub over the whole GPU matters: on a power-law graph a single
// hub's probes outnumber those of thousands of ordinary rows.
template <typename OffT, typename IndT, typename VtxT, typename OutT>
__global__ void __launch_bounds__(kSubThreads)
subset_kernel(const OffT *__restrict__ off, const IndT *__restrict__ ind,
              const VtxT *__restrict__ vertex, long long count,
              OutT *__restrict__ out)
{
    __shared__ long long s_keys[kSubSlots];
    __shared__ unsigned long long s_sum;
    auto block = cg::this_thread_block();
    auto warp = cg::tiled_partition<32>(block);
    const int wid = warp.meta_group_rank(), lane = warp.thread_rank();
    constexpr int nwarps = kSubThreads / 32;
    for (long long k = blockIdx.x; k < count; k += gridDim.x) {
        const long long v = (long long)vertex[k];
        const long long vb = off[v], ve = off[v + 1], dv = ve - vb;
        if (dv > kSubHubMin) {
            if (threadIdx.x == 0) out[k] = 0;
            continue;                              // uniform across the block
        }
        if (threadIdx.x == 0) s_sum = 0;
        int log2t = 5;
        while ((1ll << log2t) < 2 * dv) ++log2t;
        const unsigned int mask = (1u << log2t) - 1;
        for (int i = threadIdx.x; i <= (int)mask; i += kSubThreads) s_keys[i] = -1;
        __syncthreads();
        for (long long i = threadIdx.x; i < dv; i += kSubThreads) {
            const long long key = (long long)ind[vb + i];
            unsigned int slot = hash_slot((int)key, log2t);
            while (true) {
                unsigned long long prev = atomicCAS((unsigned long long *)&s_keys[slot],
                                                    (unsigned long long)-1ll,
                                                    (unsigned long long)key);
                if (prev == (unsigned long long)-1ll) break;
                slot = (slot + 1) & mask;
            }
        }
        __syncthreads();
        unsigned long long acc = 0;
        if (dv >= 2) {
            // warps take neighbours u in turn
            for (long long e = vb + wid; e < ve; e += nwarps) {
                const long long u = (long long)ind[e];
                const long long ub = off[u], ue = off[u + 1], du = ue - ub;
                if (u == v || du < 2) continue;
                if (du <= 4 * dv) {
                    for (long long i0 = lane; i0 < du; i0 += 128) {
                        long long wv[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const long long i = i0 + 32 * j;
                            wv[j] = i < du ? (long long)ind[ub + i] : -1;
                        }
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            if (wv[j] < 0) continue;
                            unsigned int slot = hash_slot((int)wv[j], log2t);
                            while (true) {
                                const long long kk = s_keys[slot];
                                if (kk == wv[j]) { ++acc; break; }
                                if (kk == -1) break;
                                slot = (slot + 1) & mask;
                            }
                        }
                    }
                } else {
                    acc += search_shorter(ind, vb, dv, ub, du, lane);
                }
            }
        }
        const unsigned long long ws = cg::reduce(warp, acc, cg::plus<unsigned long long>());
        if (lane == 0 && ws) atomicAdd(&s_sum, ws);
        __syncthreads();
        if (threadIdx.x == 0) out[k] = (OutT)s_sum;
        __syncthreads();
    }
}

template <typename OffT, typename IndT, typename VtxT, typename OutT>
__global__ void __launch_bounds__(kSubHubThreads, 1)
subset_hub_kernel(const OffT *__restrict__ off, const IndT *__restrict__ ind,
                  const VtxT *__restrict__ vertex, long long count,
                  OutT *__restrict__ out)
{
    extern __shared__ unsigned int s_bits[];          // kSubHubBits / 32 words
    __shared__ long long s_hub[kSubHubThreads];
    __shared__ int s_nhub;
    __shared__ long long s_lo, s_hi;
    __shared__ unsigned long long s_sum;
    constexpr int kBigRows = 64, kSplit = 2048, kPiece = 1024;
    __shared__ long long s_big_b[kBigRows], s_big_e[kBigRows];
    __shared__ int s_nbig;
    auto block = cg::this_thread_block();
    auto warp = cg::tiled_partition<32>(block);
    const int wid = warp.meta_group_rank(), lane = warp.thread_rank();
    constexpr int nwarps = kSubHubThreads / 32;
    const long long stride = (long long)gridDim.x * nwarps;   // neighbours per worker step
    // the listed vertices are scanned a chunk at a time, every thread
    // testing one; the hubs found are then taken one after another
    for (long long c0 = 0; c0 < count; c0 += kSubHubThreads) {
        if (threadIdx.x == 0) s_nhub = 0;
        __syncthreads();
        const long long kk = c0 + threadIdx.x;
        if (kk < count) {
            const long long v = (long long)vertex[kk];
            if ((long long)off[v + 1] - (long long)off[v] > kSubHubMin)
                s_hub[atomicAdd(&s_nhub, 1)] = kk;
        }
        __syncthreads();
        const int nh = s_nhub;
        for (int h = 0; h < nh; ++h) {
            const long long k = s_hub[h];
            const long long v = (long long)vertex[k];
            const long long vb = off[v], ve = off[v + 1], dv = ve - vb;
            // the row's id span (rows are sorted, but the bitmap must not
            // depend on it)
            long long lo = LLONG_MAX, hi = LLONG_MIN;
            for (long long i = vb + threadIdx.x; i < ve; i += kSubHubThreads) {
                const long long x = (long long)ind[i];
                lo = min(lo, x);
                hi = max(hi, x);
            }
            lo = cg::reduce(warp, lo, cg::less<long long>());
            hi = cg::reduce(warp, hi, cg::greater<long long>());
            if (threadIdx.x == 0) { s_lo = LLONG_MAX; s_hi = LLONG_MIN; s_sum = 0; s_nbig = 0; }
            __syncthreads();
            if (lane == 0) { atomicMin(&s_lo, lo); atomicMax(&s_hi, hi); }
            __syncthreads();
            lo = s_lo;
            hi = s_hi;
            const unsigned long long span = (unsigned long long)(hi - lo) + 1ull;
            const bool use_bits = span <= (unsigned long long)kSubHubBits;
            if (use_bits) {
                const int words = (int)((span + 31) >> 5);
                for (int i = threadIdx.x; i < words; i += kSubHubThreads) s_bits[i] = 0;
                __syncthreads();
                for (long long i = vb + threadIdx.x; i < ve; i += kSubHubThreads) {
                    const unsigned long long x = (unsigned long long)((long long)ind[i] - lo);
                    atomicOr(&s_bits[x >> 5], 1u << (x & 31));
                }
                __syncthreads();
            }
            unsigned long long acc = 0;
            auto sweep = [&](long long b0, long long b1) {
                // four loads in flight per lane
                for (long long i0 = b0; i0 < b1; i0 += 128) {
                    long long x[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const long long i = i0 + j * 32 + lane;
                        x[j] = i < b1 ? (long long)ind[i] - lo : -1;
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if ((unsigned long long)x[j] < span)
                            acc += (s_bits[x[j] >> 5] >> (x[j] & 31)) & 1u;
                }
            };
            for (long long e = vb + blockIdx.x + (long long)gridDim.x * wid; e < ve; e += stride) {
                const long long u = (long long)ind[e];
                const long long ub = off[u], ue = off[u + 1], du = ue - ub;
                if (u == v || du < 2) continue;
                if (use_bits && du > kSplit) {
                    // a long row is shared by the block's warps after this loop
                    int at = 0;
                    if (lane == 0) at = atomicAdd(&s_nbig, 1);
                    at = warp.shfl(at, 0);
                    if (at < kBigRows) {
                        if (lane == 0) { s_big_b[at] = ub; s_big_e[at] = ue; }
                        continue;
                    }
                }
                if (use_bits) {
                    // four loads in flight per lane
                    for (long long i0 = ub; i0 < ue; i0 += 128) {
                        long long x[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const long long i = i0 + j * 32 + lane;
                            x[j] = i < ue ? (long long)ind[i] - lo : -1;
                        }
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if ((unsigned long long)x[j] < span)
                                acc += (s_bits[x[j] >> 5] >> (x[j] & 31)) & 1u;
                    }
                } else {
                    acc += search_shorter(ind, vb, dv, ub, du, lane);
                }
            }
            if (use_bits) {
                __syncthreads();
                const int nbig = min(s_nbig, kBigRows);
                for (int r = 0; r < nbig; ++r) {
                    const long long b0 = s_big_b[r], b1 = s_big_e[r];
                    for (long long c0 = b0 + (long long)wid * kPiece; c0 < b1;
                         c0 += (long long)nwarps * kPiece)
                        sweep(c0, c0 + kPiece < b1 ? c0 + kPiece : b1);
                }
            }
            const unsigned long long ws = cg::reduce(warp, acc, cg::plus<unsigned long long>());
            if (lane == 0 && ws) atomicAdd(&s_sum, ws);
            __syncthreads();
            if (threadIdx.x == 0 && s_sum) add_out(&out[k], s_sum);
            __syncthreads();                       // s_bits, s_lo and s_sum are reused
        }
        __syncthreads();                           // every thread has read s_nhub
    }
}

template <typename OffT, typename IndT, typename VtxT, typename OutT>
gtc_status launch_subset(const OffT *off, const IndT *ind, const VtxT *vertex,
                         long long count, OutT *out, cudaStream_t stream)
{
    if (count <= 0) return GTC_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long blocks = count < (long long)sms * 8 ? count : (long long)sms * 8;
    subset_kernel<OffT, IndT, VtxT, OutT><<<(unsigned)blocks, kSubThreads, 0, stream>>>(
        off, ind, vertex, count, out);
    // the hub kernel adds to what subset_kernel wrote (0 for hubs), in
    // stream order
    auto hub = subset_hub_kernel<OffT, IndT, VtxT, OutT>;
    const int smem = (int)(kSubHubBits / 8);
    if (cudaFuncSetAttribute(hub, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        return GTC_ERR_CUDA;
    hub<<<(unsigned)sms, kSubHubThreads, smem, stream>>>(off, ind, vertex, count, out);
    return cudaGetLastError() == cudaSuccess ? GTC_OK : GTC_ERR_CUDA;
}

// ================================================================== compat

// int64 neighbour ids -> int32.  An id outside [0, nv) becomes -1, which the
// counting kernels flag (kErrIndexRange) and skip, so a wide id can never
// wrap into a valid-looking one.
__global__ void narrow_kernel(const long long *__restrict__ in, int *__restrict__ out,
                              long long count, long long nv)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const long long x = in[i];
        out[i] = (x >= 0 && x < nv) ? (int)x : -1;
    }
}

__global__ void narrow_out_kernel(const long long *__restrict__ in, int *__restrict__ out,
                                  long long count)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (int)in[i];
}

struct CompatCache {
    void *ptr = nullptr;
    size_t bytes = 0;
};
std::mutex g_compat_mu;
CompatCache g_compat[64];
thread_local gtc_status g_compat_status = GTC_OK;
// Workspace of this thread's last kernelCall shim that launched a count
// (its status word is read by gtc_compat_last_status), or null.
thread_local const void *g_compat_ws = nullptr;

// Device error bits -> status.
gtc_status status_from_bits(unsigned int bits)
{
    return (bits & kErrIndexRange) ? GTC_ERR_INVALID_CSR : GTC_OK;
}

void *compat_workspace(size_t bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_compat_mu);
    CompatCache &c = g_compat[dev];
    if (c.bytes < bytes) {
        if (c.ptr) cudaFree(c.ptr);
        c.ptr = nullptr;
        c.bytes = 0;
        if (cudaMalloc(&c.ptr, bytes) != cudaSuccess) { c.ptr = nullptr; return nullptr; }
        c.bytes = bytes;
    }
    return c.ptr;
}

// Largest degree of a CSR into *out (zeroed by the caller); grid-stride,
// warp max, one atomic per warp.
template <typename OffT>
__global__ void max_degree_kernel(const OffT *__restrict__ off, long long n,
                                  unsigned long long *out)
{
    unsigned long long best = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const long long d = (long long)off[v + 1] - (long long)off[v];
        if (d > 0 && (unsigned long long)d > best) best = (unsigned long long)d;
    }
    best = cg::reduce(cg::tiled_partition<32>(cg::this_thread_block()), best,
                      cg::greater<unsigned long long>());
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

// Skew above which the compat shims switch a low-mean-degree graph from
// vertex-id to degree-rank labels: R-MAT scale 20-22 at edge factor 6-8 (skew
// in the thousands) count 15-25% faster with ranks, while meshes and ER
// graphs (skew below 4) are faster with ids.
constexpr long long kCompatSkewRanks = 64;

// The compat shims' launch shape: the mean-degree rule, then -- since these
// calls synchronise anyway -- one read of the largest degree, and rank labels
// for a skewed graph.  scratch: 8 bytes of device memory.
template <typename OffT>
RowConfig compat_row_config(const OffT *d_off, long long n, long long nnz, void *scratch)
{
    RowConfig cfg = pick_row_config(n, nnz);
    if (cfg.rank_labels || n <= 0 || nnz <= 0) return cfg;
    unsigned long long *dmax = static_cast<unsigned long long *>(scratch);
    unsigned long long h = 0;
    if (cudaMemsetAsync(dmax, 0, sizeof(*dmax), 0) != cudaSuccess) return cfg;
    const long long want = div_up<long long>(n, 256);
    max_degree_kernel<OffT><<<(unsigned)(want < 1184 ? want : 1184), 256>>>(d_off, n, dmax);
    if (cudaMemcpy(&h, dmax, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return cfg;
    if ((long long)h * n > kCompatSkewRanks * nnz) {
        cfg.rank_labels = true;
        cfg.merge_rows = false;
    }
    return cfg;
}

bool compat_block_size_ok(unsigned int bs)
{
    switch (bs) {
    case 32: case 64: case 96: case 128: case 192: case 256: case 512: case 1024: return true;
    default: return false;
    }
}

}  // namespace
}  // namespace gtc

using namespace gtc;

extern "C" {

const char *gtc_status_string(gtc_status s)
{
    switch (s) {
    case GTC_OK: return "ok";
    case GTC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case GTC_ERR_INVALID_CSR: return "invalid CSR";
    case GTC_ERR_WORKSPACE_TOO_SMALL: return "workspace too small";
    case GTC_ERR_CUDA: return "CUDA runtime error";
    case GTC_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GTC_ERR_UNSUPPORTED: return "unsupported device or configuration";
    case GTC_ERR_TIMEOUT: return "bounded device wait timed out";
    case GTC_ERR_CAPACITY: return "capacity exceeded";
    case GTC_ERR_BUSY: return "busy";
    }
    return "unknown status";
}

gtc_status gtc_device_info(int *sm_count, int *cc)
{
    if (!sm_count || !cc) return GTC_ERR_INVALID_ARGUMENT;
    int dev = 0, major = 0, minor = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GTC_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess)
        return GTC_ERR_CUDA;
    *sm_count = sms;
    *cc = major * 10 + minor;
    return GTC_OK;
}

gtc_status gtc_workspace_size(int64_t n, int64_t nnz, int off_bits, gtc_mode mode, size_t *bytes)
{
    if (!bytes || n < 0 || nnz < 0 || (off_bits != 32 && off_bits != 64)) return GTC_ERR_INVALID_ARGUMENT;
    if (mode != GTC_MODE_PLAIN && mode != GTC_MODE_ORIENTED) return GTC_ERR_INVALID_ARGUMENT;
    if (n > 0x7fffffffll) return GTC_ERR_UNSUPPORTED;           // int32 vertex ids
    if (off_bits == 32 && nnz > 0x7fffffffll) return GTC_ERR_INVALID_ARGUMENT;
    *bytes = make_plan(n, nnz, off_bits, mode == GTC_MODE_PLAIN).bytes;
    return GTC_OK;
}

gtc_status gtc_count_launches(int64_t n, int64_t nnz, gtc_mode mode,
                              const gtc_tuning *tuning, int *launches, int *labels)
{
    if (n < 0 || nnz < 0 || !launches || !labels ||
        (mode != GTC_MODE_PLAIN && mode != GTC_MODE_ORIENTED))
        return GTC_ERR_INVALID_ARGUMENT;
    RowConfig cfg = pick_row_config(n, nnz);
    const gtc_status st = apply_tuning(cfg, tuning);
    if (st != GTC_OK) return st;
    *launches = launches_per_count(cfg, mode == GTC_MODE_PLAIN, n);
    *labels = cfg.rank_labels ? GTC_LABELS_DEGREE_RANK : GTC_LABELS_VERTEX_ID;
    return GTC_OK;
}

gtc_status gtc_count_tuned(const void *d_off, int off_bits, const int32_t *d_ind, int64_t n,
                           int64_t nnz, gtc_mode mode, int64_t *d_r, int64_t *d_t,
                           double *d_lcc, int64_t *d_global, void *d_workspace, size_t ws_bytes,
                           gtc_stream_t stream, const gtc_tuning *tuning)
{
    size_t need = 0;
    gtc_status st = gtc_workspace_size(n, nnz, off_bits, mode, &need);
    if (st != GTC_OK) return st;
    if (!d_off || (nnz > 0 && !d_ind) || !d_workspace) return GTC_ERR_INVALID_ARGUMENT;
    if (mode == GTC_MODE_ORIENTED && (d_r || d_t || d_lcc)) return GTC_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_workspace) & 255) return GTC_ERR_INVALID_ARGUMENT;
    if (ws_bytes < need) return GTC_ERR_WORKSPACE_TOO_SMALL;
    const bool pv = mode == GTC_MODE_PLAIN;
    RowConfig cfg = pick_row_config(n, nnz);
    st = apply_tuning(cfg, tuning);
    if (st != GTC_OK) return st;
    long long *r = reinterpret_cast<long long *>(d_r);
    long long *t = reinterpret_cast<long long *>(d_t);
    long long *g = reinterpret_cast<long long *>(d_global);
    if (off_bits == 32)
        return run_count<int>(static_cast<const int *>(d_off), d_ind, n, nnz, pv, r, t, d_lcc, g,
                              d_workspace, ws_bytes, as_stream(stream), cfg, nullptr);
    return run_count<long long>(static_cast<const long long *>(d_off), d_ind, n, nnz, pv, r, t,
                                d_lcc, g, d_workspace, ws_bytes, as_stream(stream), cfg, nullptr);
}

gtc_status gtc_count(const void *d_off, int off_bits, const int32_t *d_ind, int64_t n,
                     int64_t nnz, gtc_mode mode, int64_t *d_r, int64_t *d_t, double *d_lcc,
                     int64_t *d_global, void *d_workspace, size_t ws_bytes, gtc_stream_t stream)
{
    return gtc_count_tuned(d_off, off_bits, d_ind, n, nnz, mode, d_r, d_t, d_lcc, d_global,
                           d_workspace, ws_bytes, stream, nullptr);
}

gtc_status gtc_count_phase_times(const void *d_off, int off_bits, const int32_t *d_ind,
                                 int64_t n, int64_t nnz, void *d_workspace, size_t ws_bytes,
                                 float *h_ms, const gtc_tuning *tuning)
{
    size_t need = 0;
    gtc_status st = gtc_workspace_size(n, nnz, off_bits, GTC_MODE_PLAIN, &need);
    if (st != GTC_OK) return st;
    if (!d_off || (nnz > 0 && !d_ind) || !d_workspace || !h_ms) return GTC_ERR_INVALID_ARGUMENT;
    if (ws_bytes < need) return GTC_ERR_WORKSPACE_TOO_SMALL;
    RowConfig cfg = pick_row_config(n, nnz);
    st = apply_tuning(cfg, tuning);
    if (st != GTC_OK) return st;
    CountTimings tm;
    for (int i = 0; i < 5; ++i)
        if (cudaEventCreate(&tm.ev[i]) != cudaSuccess) return GTC_ERR_CUDA;
    if (off_bits == 32)
        st = run_count<int>(static_cast<const int *>(d_off), d_ind, n, nnz, true, nullptr,
                            nullptr, nullptr, nullptr, d_workspace, ws_bytes, 0, cfg, &tm);
    else
        st = run_count<long long>(static_cast<const long long *>(d_off), d_ind, n, nnz, true,
                                  nullptr, nullptr, nullptr, nullptr, d_workspace, ws_bytes, 0,
                                  cfg, &tm);
    if (st == GTC_OK && cudaEventSynchronize(tm.ev[4]) != cudaSuccess) st = GTC_ERR_CUDA;
    if (st == GTC_OK && n > 0) {
        for (int i = 0; i < 4; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, tm.ev[i], tm.ev[i + 1]);
            h_ms[i] = ms;
        }
    }
    for (int i = 0; i < 5; ++i) cudaEventDestroy(tm.ev[i]);
    return st;
}

size_t gtc_validate_workspace_size(int64_t n, int64_t nnz)
{
    (void)n;
    (void)nnz;
    return 256;
}

gtc_status gtc_validate_csr(const void *d_off, int off_bits, const int32_t *d_ind, int64_t n,
                            int64_t nnz, void *d_workspace, size_t ws_bytes, int32_t *h_reason,
                            gtc_stream_t stream)
{
    if (!d_off || (nnz > 0 && !d_ind) || !d_workspace || !h_reason || n < 0 || nnz < 0)
        return GTC_ERR_INVALID_ARGUMENT;
    if (off_bits != 32 && off_bits != 64) return GTC_ERR_INVALID_ARGUMENT;
    if (n > 0x7fffffffll) return GTC_ERR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(d_workspace) & 255) return GTC_ERR_INVALID_ARGUMENT;
    if (ws_bytes < gtc_validate_workspace_size(n, nnz)) return GTC_ERR_WORKSPACE_TOO_SMALL;
    if (off_bits == 32)
        return run_validate<int>(static_cast<const int *>(d_off), d_ind, n, nnz, d_workspace,
                                 h_reason, as_stream(stream));
    return run_validate<long long>(static_cast<const long long *>(d_off), d_ind, n, nnz,
                                   d_workspace, h_reason, as_stream(stream));
}

gtc_status gtc_count_subset(const void *d_off, int off_bits, const int32_t *d_ind,
                            const int32_t *d_vertex, int64_t count, int64_t *d_out,
                            gtc_stream_t stream)
{
    if (count < 0) return GTC_ERR_INVALID_ARGUMENT;
    if (count == 0) return GTC_OK;
    if (!d_off || !d_ind || !d_vertex || !d_out) return GTC_ERR_INVALID_ARGUMENT;
    if (off_bits == 32)
        return launch_subset(static_cast<const int *>(d_off), d_ind, d_vertex, count,
                             reinterpret_cast<long long *>(d_out), as_stream(stream));
    if (off_bits == 64)
        return launch_subset(static_cast<const long long *>(d_off), d_ind, d_vertex, count,
                             reinterpret_cast<long long *>(d_out), as_stream(stream));
    return GTC_ERR_INVALID_ARGUMENT;
}

gtc_status gtc_compat_last_status(void)
{
    if (g_compat_status != GTC_OK || !g_compat_ws) return g_compat_status;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GTC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_compat_mu);
    // the cached workspace was replaced by a later, larger call: its status
    // word belonged to that call
    if (g_compat[dev].ptr != g_compat_ws) return g_compat_status;
    unsigned int bits = 0;
    // a copy on the legacy default stream, so it waits for the count
    if (cudaMemcpy(&bits, g_compat_ws, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess)
        return GTC_ERR_CUDA;
    return status_from_bits(bits);
}

gtc_status gtc_count_status(const void *d_workspace, size_t ws_bytes, gtc_stream_t stream,
                            uint32_t *h_bits)
{
    if (!d_workspace || ws_bytes < sizeof(unsigned int)) return GTC_ERR_INVALID_ARGUMENT;
    unsigned int bits = 0;
    cudaStream_t s = as_stream(stream);
    if (cudaMemcpyAsync(&bits, d_workspace, sizeof(bits), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return GTC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return GTC_ERR_CUDA;
    if (h_bits) *h_bits = bits;
    return status_from_bits(bits);
}

gtc_status gtc_compat_release(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GTC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_compat_mu);
    CompatCache &c = g_compat[dev];
    if (c.ptr) cudaFree(c.ptr);
    c.ptr = nullptr;
    c.bytes = 0;
    return GTC_OK;
}

void gtc_kernelCall_i64(unsigned int numberBlocks, unsigned int numberThreads, int64_t nv,
                        const int64_t *d_off, const int64_t *d_ind, int64_t *out,
                        int64_t threads_per_block, int64_t number_blocks, int64_t shifter)
{
    (void)numberBlocks; (void)threads_per_block; (void)number_blocks; (void)shifter;
    g_compat_status = GTC_OK;
    g_compat_ws = nullptr;
    if (!compat_block_size_ok(numberThreads)) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    if (nv <= 0 || !d_off || !out) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    int64_t nnz = 0;
    // the pipeline needs nnz = off[nv]: one 8-byte read on the legacy stream
    if (cudaMemcpy(&nnz, d_off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
        g_compat_status = GTC_ERR_CUDA;
        return;
    }
    if (nnz < 0 || nv > 0x7fffffffll) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    size_t need = make_plan(nv, nnz, 64, true).bytes;
    size_t ind_bytes = (((size_t)nnz * sizeof(int)) + 255) & ~(size_t)255;
    char *ws = static_cast<char *>(compat_workspace(need + ind_bytes + 256));
    if (!ws) { g_compat_status = GTC_ERR_OUT_OF_MEMORY; return; }
    int *ind32 = reinterpret_cast<int *>(ws + need);
    if (nnz > 0)
        narrow_kernel<<<(unsigned)div_up<long long>(nnz, 256), 256>>>(
            reinterpret_cast<const long long *>(d_ind), ind32, nnz, nv);
    RowConfig cfg = compat_row_config(reinterpret_cast<const long long *>(d_off), nv, nnz,
                                      ws + need + ind_bytes);
    g_compat_status = run_count<long long>(reinterpret_cast<const long long *>(d_off), ind32, nv,
                                           nnz, true, reinterpret_cast<long long *>(out), nullptr,
                                           nullptr, nullptr, ws, need, 0, cfg, nullptr);
    if (g_compat_status == GTC_OK) g_compat_ws = ws;
}

void gtc_kernelCall_i32(unsigned int numberBlocks, unsigned int numberThreads, int32_t nv,
                        const int32_t *d_off, const int32_t *d_ind, int32_t *out,
                        int32_t threads_per_block, int32_t number_blocks, int32_t shifter)
{
    (void)numberBlocks; (void)threads_per_block; (void)number_blocks; (void)shifter;
    g_compat_status = GTC_OK;
    g_compat_ws = nullptr;
    if (!compat_block_size_ok(numberThreads)) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    if (nv <= 0 || !d_off || !out) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    int32_t nnz = 0;
    if (cudaMemcpy(&nnz, d_off + nv, sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
        g_compat_status = GTC_ERR_CUDA;
        return;
    }
    if (nnz < 0) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    size_t need = make_plan(nv, nnz, 32, true).bytes;
    size_t r_bytes = (((size_t)nv * sizeof(long long)) + 255) & ~(size_t)255;
    char *ws = static_cast<char *>(compat_workspace(need + r_bytes + 256));
    if (!ws) { g_compat_status = GTC_ERR_OUT_OF_MEMORY; return; }
    long long *r64 = reinterpret_cast<long long *>(ws + need);
    RowConfig cfg = compat_row_config(d_off, nv, nnz, ws + need + r_bytes);
    g_compat_status = run_count<int>(d_off, d_ind, nv, nnz, true, r64, nullptr, nullptr, nullptr,
                                     ws, need, 0, cfg, nullptr);
    if (g_compat_status == GTC_OK) {
        narrow_out_kernel<<<(unsigned)div_up<long long>(nv, 256), 256>>>(r64, out, nv);
        g_compat_ws = ws;
    }
}

void gtc_kernelCall_vertex_i64(unsigned int numberBlocks, unsigned int numberThreads, int64_t nv,
                               const int64_t *vertex, const int64_t *d_off, const int64_t *d_ind,
                               int64_t *out, int64_t threads_per_block, int64_t number_blocks,
                               int64_t shifter)
{
    (void)numberBlocks; (void)threads_per_block; (void)number_blocks; (void)shifter;
    g_compat_status = GTC_OK;
    g_compat_ws = nullptr;
    if (!compat_block_size_ok(numberThreads)) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    if (nv < 0 || (nv > 0 && (!vertex || !d_off || !d_ind || !out))) {
        g_compat_status = GTC_ERR_INVALID_ARGUMENT;
        return;
    }
    g_compat_status = launch_subset(reinterpret_cast<const long long *>(d_off),
                                    reinterpret_cast<const long long *>(d_ind),
                                    reinterpret_cast<const long long *>(vertex), nv,
                                    reinterpret_cast<long long *>(out), 0);
}

void gtc_kernelCall_vertex_i32(unsigned int numberBlocks, unsigned int numberThreads, int32_t nv,
                               const int32_t *vertex, const int32_t *d_off, const int32_t *d_ind,
                               int32_t *out, int32_t threads_per_block, int32_t number_blocks,
                               int32_t shifter)
{
    (void)numberBlocks; (void)threads_per_block; (void)number_blocks; (void)shifter;
    g_compat_status = GTC_OK;
    g_compat_ws = nullptr;
    if (!compat_block_size_ok(numberThreads)) { g_compat_status = GTC_ERR_INVALID_ARGUMENT; return; }
    if (nv < 0 || (nv > 0 && (!vertex || !d_off || !d_ind || !out))) {
        g_compat_status = GTC_ERR_INVALID_ARGUMENT;
        return;
    }
    g_compat_status = launch_subset(d_off, d_ind, vertex, (long long)nv, out, 0);
}

}  // extern "C"
