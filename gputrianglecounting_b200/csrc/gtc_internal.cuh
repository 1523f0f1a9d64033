// gtc_internal.cuh -- shared device/host helpers of the B200 triangle counter.
//
// Algorithm (same output as the reference's per-vertex kernel,
// src/clusteringCount.cu:314-359, computed differently):
//   1. order the vertices by degree -- as (degree, id) with vertex-id labels,
//      or by a counting sort into ranks with degree-rank labels -- orient
//      every undirected edge from its lower to its higher end and build the
//      forward lists N+(v) in one pass, each at the start of v's own CSR
//      segment (holding ids or ranks); lists a consumer reads in order are
//      sorted;
//   2. give every oriented edge one "apex" that intersects for it: the end
//      with the longer forward list (ties to the source), except that with
//      rank labels a block-kernel apex owns every edge to a lower-ranked
//      neighbour.  The apex's N+ is staged in shared memory (hash table, rank
//      bitmap or per-rank counters) and the partner's N+ is probed into it --
//      or, for short lists with vertex-id labels, the two id-ordered lists
//      are merged by one lane -- so each triangle {u,v,w} is found exactly
//      once, at the edge between its two lowest-ordered vertices;
//   3. credit the triangle to all three vertices: the apex through a register
//      or block count, the partner through a warp reduction or a ballot
//      popcount, the third vertex w through a shared per-member hit counter
//      flushed to global memory once per (apex, w).
// All counting is integer and exact; the result does not depend on the
// order in which blocks run, on the labels or on the order of equal degrees.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gtc_b200.h"

namespace gtc {

// ------------------------------------------------------------------ tuning
constexpr int kPrepThreads = 256;           // merge-path tile kernels
constexpr int kPrepItemsPerThread = 8;      // (rows + entries) per thread
constexpr int kPrepTile = kPrepThreads * kPrepItemsPerThread;
constexpr long long kRowPlaceThreadMin = 1ll << 18;   // rows from which a thread takes a row
constexpr int kLongRowMin = 64;             // longest row a placement thread takes

constexpr int kRowThreads = 256;            // warp-per-item count kernel
constexpr int kRowSlots = 512;              // shared table slots per warp
constexpr int kRowMinBlocks = 6;            // 48 warps per SM (register budget 42)
constexpr int kMinItemLen = 32;             // smallest warp work item (entries)
constexpr int kMaxItemLen = 32768;          // largest: a 16-bit hit counter must not carry
constexpr int kBigThreads = 256;            // block-per-row count kernel
constexpr int kBigMinBlocks = 8;            // 8 blocks (64 warps) per SM: 32 registers
constexpr int kMinBigChunk = 32;            // smallest block-kernel item (entries)
constexpr int kBigTableLog2 = 12;
constexpr int kBigTableSlots = 1 << kBigTableLog2;   // shared hash slots (block kernel)
constexpr int kBigHashMaxFdeg = 2048;       // longest list hashed (load <= 1/2)

// Degree-rank labels (skewed graphs): vertices are ordered by degree (a
// counting sort over kRankBuckets degree buckets: exact degrees below half of
// them, then a float-like map with kRankBuckets / 32 buckets per octave) and
// every forward list holds the ranks of its members, sorted ascending.
constexpr int kRankBuckets = 1 << 13;
constexpr int kRankScanThreads = 1024;
constexpr int kRankThreads = 256;           // histogram / rank kernels
constexpr int kRankChunk = 4096;            // vertices per histogram / rank block
constexpr int kSortThreads = 256;           // forward-list sort kernel (warp per 32 rows)
constexpr int kSortRegMax = 1024;           // longest list sorted in registers
constexpr int kDirectRanks = 12288;         // block kernel: one 16-bit counter per rank
constexpr int kTrimLoads = 2;               // block kernel: loads in flight per partner window
constexpr int kBitWords = 2048;             // block kernel rank bitmap: 65536 ranks
constexpr int kBitKeys = 2048;              // longest apex list on the bitmap path
constexpr int kSegBuckets = 1024;           // degree buckets per graph (batched rank labels)

// Error bits written to the workspace status word (the first 4 bytes of
// every counting workspace) by device code; gtc_count_status reads them.
enum : unsigned int {
    kErrIndexRange = 1u,   // a neighbour id outside [0, n) was met (and skipped)
};

// Per-vertex record built once per count: forward-list start, forward degree
// and the vertex's order key in one 16-byte load.  The key is the degree
// (vertex-id labels: order by (degree, id)) or the degree rank (rank labels:
// every key distinct).
struct __align__(16) VInfo {
    long long fbeg;
    int fdeg;
    int key;
};

// Order comparison: does x (key kx) come after y (key ky)?  Lexicographic in
// (key, id), which is the (degree, id) order for degree keys and the rank
// order for rank keys (distinct keys never reach the id tie-break).
__device__ __forceinline__ bool rank_above(int kx, int x, int ky, int y)
{
    return kx > ky || (kx == ky && x > y);
}

__device__ __forceinline__ unsigned int hash_slot(int key, int log2_slots)
{
    return ((unsigned int)key * 0x9E3779B1u) >> (32 - log2_slots);
}

__host__ __device__ __forceinline__ int ceil_log2(long long v)
{
    int l = 0;
    while ((1ll << l) < v) ++l;
    return l;
}

template <typename T>
__host__ __device__ __forceinline__ T div_up(T a, T b)
{
    return (a + b - 1) / b;
}

// Largest row r in [0, n) with off[r] <= e (e < off[n]): the row holding e.
template <typename OffT>
__device__ __forceinline__ long long row_of_entry(const OffT *__restrict__ off,
                                                  long long n, long long e)
{
    long long lo = 0, hi = n;           // invariant: off[lo] <= e < off[hi]
    while (hi - lo > 1) {
        long long mid = (lo + hi) >> 1;
        if ((long long)off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------ host helpers
struct Plan {
    long long n = 0, nnz = 0;
    int off_bits = 64;
    long long n_tiles = 0;       // merge-path tiles over rows + entries
    long long fwd_cap = 0;       // capacity of the forward adjacency
    // workspace byte offsets
    size_t o_status = 0, o_counters = 0, o_deg = 0, o_fcnt = 0, o_vinfo = 0, o_find = 0,
           o_tacc = 0, o_trow = 0, o_irow = 0, o_hist = 0, o_rank = 0, o_order = 0,
           o_bitem = 0, o_long = 0;
    size_t bytes = 0;
};

// Counters block in the workspace (device, zeroed at the start of a count).
struct Counters {
    unsigned long long tri_total;     // triangles found (T)
    unsigned long long row_items;     // dynamic item queue, group kernel
    unsigned long long big_items;     // dynamic item queue, block kernel
    unsigned long long big_rows;      // number of rows for the block kernel
    unsigned long long sort_groups;   // dynamic queue of 32-row groups, list sort
    unsigned long long big_total;     // block-kernel items posted by the forward build
    unsigned long long long_rows;     // rows the per-warp row placement leaves to blocks
    unsigned long long long_next;     // dynamic queue over those rows
};


// out[0..count) = exclusive prefix of in, out[count] = total (in may be out);
// tmp holds scan_tmp_bytes(count) bytes.
size_t scan_tmp_bytes(long long count);
cudaError_t exclusive_scan_i64(const long long *in, long long *out,
                               long long count, void *tmp,
                               cudaStream_t stream);

}  // namespace gtc
