// gtc_scan.cu -- device-wide exclusive prefix sum of int64 values
// (reduce, scan of the block sums, scan + add), used for the per-graph
// degree-bucket histogram of batched degree-rank labels.
#include "gtc_internal.cuh"

namespace gtc {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kItems = 8;
constexpr int kChunk = kScanThreads * kItems;

__device__ __forceinline__ long long warp_incl_scan(long long v)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        long long o = __shfl_up_sync(0xffffffffu, v, d);
        if ((threadIdx.x & 31) >= d) v += o;
    }
    return v;
}

// Exclusive scan of one value per thread across the block; returns the
// thread's exclusive prefix and writes the block total to *total.
__device__ long long block_excl_scan(long long v, long long *total)
{
    __shared__ long long warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long incl = warp_incl_scan(v);
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        long long s = (lane < kScanThreads / 32) ? warp_sums[lane] : 0;
        s = warp_incl_scan(s);
        if (lane < kScanThreads / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    long long base = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return base + incl - v;
}

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const long long *__restrict__ in, long long count,
                   long long *__restrict__ partials)
{
    long long base = (long long)blockIdx.x * kChunk + (long long)threadIdx.x * kItems;
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < count) s += in[base + k];
    long long total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// One block scans the partials in place (exclusive), chunk by chunk.
__global__ void __launch_bounds__(kScanThreads)
scan_partials_kernel(long long *partials, long long count)
{
    long long carry = 0;
    for (long long c0 = 0; c0 < count; c0 += kChunk) {
        long long base = c0 + (long long)threadIdx.x * kItems;
        long long v[kItems];
        long long s = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            v[k] = (base + k < count) ? partials[base + k] : 0;
            s += v[k];
        }
        long long total;
        long long ex = block_excl_scan(s, &total) + carry;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (base + k < count) partials[base + k] = ex;
            ex += v[k];
        }
        carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads)
scan_apply_kernel(const long long *in, long long *out, long long count,
                  const long long *__restrict__ partials, int write_total)
{
    long long base = (long long)blockIdx.x * kChunk + (long long)threadIdx.x * kItems;
    long long v[kItems];
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        v[k] = (base + k < count) ? in[base + k] : 0;
        s += v[k];
    }
    long long total;
    long long ex = block_excl_scan(s, &total) + partials[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (base + k < count) out[base + k] = ex;
        ex += v[k];
    }
    if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1)
        out[count] = ex;
}

}  // namespace

size_t scan_tmp_bytes(long long count)
{
    long long blocks = div_up<long long>(count > 0 ? count : 1, kChunk);
    return (size_t)(blocks + 1) * sizeof(long long);
}

// out[0..count) = exclusive prefix of in, out[count] = total.  `in` and `out`
// may be the same array.  tmp must hold scan_tmp_bytes(count).
cudaError_t exclusive_scan_i64(const long long *in, long long *out,
                               long long count, void *tmp, cudaStream_t stream)
{
    if (count <= 0) {
        return cudaMemsetAsync(out, 0, sizeof(long long), stream);
    }
    long long blocks = div_up<long long>(count, kChunk);
    long long *partials = static_cast<long long *>(tmp);
    scan_reduce_kernel<<<(unsigned)blocks, kScanThreads, 0, stream>>>(in, count, partials);
    scan_partials_kernel<<<1, kScanThreads, 0, stream>>>(partials, blocks);
    scan_apply_kernel<<<(unsigned)blocks, kScanThreads, 0, stream>>>(in, out, count, partials, 1);
    return cudaGetLastError();
}

}  // namespace gtc
