// gtc_core.cu -- the single-graph counting pipeline: forward-list build
// (merge-path tiles over rows + entries), apex/partner intersection kernels
// and the exact epilogue (r = 2t, lcc, global count).
//
// Reference operator replaced: count_all_trianglesGPU<T,bs> + kernelCall<T>
// (src/clusteringCount.cu:314-359, :415-467) and the thrust::reduce global
// sum (src/gpurun.cu:40).
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <nvtx3/nvToolsExt.h>
#include <type_traits>

#include "gtc_core.cuh"

namespace cg = cooperative_groups;

namespace gtc {

// ======================================================= forward-list build

__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

// Monotone map of a degree onto B buckets (B a power of two >= 64): exact
// below B/2, then B/32 buckets per octave -- a float with log2(B/32)
// mantissa bits -- for the next 16 octaves, the rest in the last bucket.
// Degrees that share a bucket above B/2 differ by less than a factor
// 2^(32/B), so the hubs of a skewed graph stay in degree order (a linear map
// put every degree >= B-1 into one bucket, in arbitrary order, which left the
// largest hubs' forward lists long).
template <int B>
__device__ __forceinline__ int degree_bucket(int d)
{
    constexpr int kExact = B / 2, kPer = B / 32;
    constexpr int kLe = ilog2(kExact), kMb = ilog2(kPer);
    if (d < kExact) return d < 0 ? 0 : d;
    const int l = 31 - __clz(d);
    const int b = kExact + (l - kLe) * kPer + ((d >> (l - kMb)) & (kPer - 1));
    return b < B ? b : B - 1;
}

__device__ __forceinline__ int rank_bucket(int d) { return degree_bucket<kRankBuckets>(d); }

// Degree of vertex v (0 past the end).
__device__ __forceinline__ int vertex_degree(const void *off_v, int off_bits, long long n,
                                             long long v)
{
    if (v >= n) return 0;
    if (off_bits == 32) {
        const int *off = static_cast<const int *>(off_v);
        return off[v + 1] - off[v];
    }
    const long long *off = static_cast<const long long *>(off_v);
    return (int)(off[v + 1] - off[v]);
}

// Count this block's kRankChunk vertices per degree bucket in shared memory
// (warp-aggregated); v = base + k * kRankThreads + threadIdx.x.
template <class Bucket>
__device__ __forceinline__ void chunk_bucket_counts(unsigned int *cnt, long long n,
                                                    const Bucket &bucket_of)
{
    for (int k = threadIdx.x; k < kRankBuckets; k += kRankThreads) cnt[k] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kRankChunk;
    const int lane = threadIdx.x & 31;
#pragma unroll 4
    for (int k = 0; k < kRankChunk / kRankThreads; ++k) {
        const long long v = base + k * kRankThreads + threadIdx.x;
        const unsigned int b = v < n ? (unsigned int)bucket_of(v) : 0xffffffffu;
        const unsigned int peers = __match_any_sync(0xffffffffu, b);
        if (v < n && lane == __ffs(peers) - 1) atomicAdd(&cnt[b], (unsigned int)__popc(peers));
    }
    __syncthreads();
}

// deg[v] and the degree-bucket histogram (rank labels): each block counts
// kRankChunk vertices in shared memory and adds its non-zero buckets.
__global__ void __launch_bounds__(kRankThreads)
degree_hist_kernel(const void *off_v, int off_bits, long long n, int *__restrict__ deg,
                   unsigned long long *__restrict__ hist)
{
    __shared__ unsigned int cnt[kRankBuckets];
    chunk_bucket_counts(cnt, n, [&](long long v) {
        const int d = vertex_degree(off_v, off_bits, n, v);
        deg[v] = d;
        return rank_bucket(d);
    });
    for (int k = threadIdx.x; k < kRankBuckets; k += kRankThreads)
        if (cnt[k]) atomicAdd(&hist[k], (unsigned long long)cnt[k]);
}

// Exclusive scan of the degree-bucket histogram, in place (one block; each
// thread owns kRankBuckets / kRankScanThreads consecutive buckets).
__global__ void __launch_bounds__(kRankScanThreads)
rank_scan_kernel(unsigned long long *__restrict__ hist)
{
    constexpr int kPer = kRankBuckets / kRankScanThreads;
    __shared__ unsigned long long warp_sum[kRankScanThreads / 32];
    unsigned long long h[kPer];
    unsigned long long mine = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        h[k] = hist[threadIdx.x * kPer + k];
        mine += h[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    unsigned long long run = incl - mine;
    for (int i = 0; i < warp; ++i) run += warp_sum[i];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        hist[threadIdx.x * kPer + k] = run;
        run += h[k];
    }
}

// rank[v]: position of v in degree order (bucket start + arrival in the
// bucket; ties between equal degrees fall in any order, which changes which
// endpoint owns an edge but never a count); order[rank] = v.  Each block
// reserves one range per non-zero bucket for its kRankChunk vertices, then
// hands out positions from shared memory.
__global__ void __launch_bounds__(kRankThreads)
rank_kernel(const int *__restrict__ deg, long long n, unsigned long long *__restrict__ cursor,
            int *__restrict__ rank, int *__restrict__ order)
{
    __shared__ unsigned int cnt[kRankBuckets];
    chunk_bucket_counts(cnt, n, [&](long long v) { return rank_bucket(deg[v]); });
    for (int k = threadIdx.x; k < kRankBuckets; k += kRankThreads)
        if (cnt[k]) cnt[k] = (unsigned int)atomicAdd(&cursor[k], (unsigned long long)cnt[k]);
    __syncthreads();
    const long long base = (long long)blockIdx.x * kRankChunk;
    const int lane = threadIdx.x & 31;
#pragma unroll 4
    for (int k = 0; k < kRankChunk / kRankThreads; ++k) {
        const long long v = base + k * kRankThreads + threadIdx.x;
        const unsigned int b = v < n ? (unsigned int)rank_bucket(deg[v]) : 0xffffffffu;
        const unsigned int peers = __match_any_sync(0xffffffffu, b);
        const int leader = __ffs(peers) - 1;
        unsigned int at = 0;
        if (v < n && lane == leader) at = atomicAdd(&cnt[b], (unsigned int)__popc(peers));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (v < n) {
            const int r = (int)(at + __popc(peers & ((1u << lane) - 1u)));
            rank[v] = r;
            order[r] = (int)v;
        }
    }
}

// ---- graph-major degree ranks of a batch (SegRanks)

// Graph holding vertex v: the largest g < G with vstart[g] <= v.
__device__ __forceinline__ long long seg_of(const long long *__restrict__ vstart, long long G,
                                            long long v)
{
    long long lo = 0, hi = G;
    while (hi - lo > 1) {
        const long long mid = (lo + hi) >> 1;
        if (vstart[mid] <= v) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ long long seg_key(const long long *__restrict__ vstart, long long G,
                                             long long v, int d)
{
    return seg_of(vstart, G, v) * kSegBuckets + degree_bucket<kSegBuckets>(d);
}

// deg[v] and the per-graph degree-bucket histogram ghist[g * kSegBuckets + b]
// (warp-aggregated global atomics).
template <typename OffT>
__global__ void seg_degree_hist_kernel(const OffT *__restrict__ off, long long n,
                                       const long long *__restrict__ vstart, long long G,
                                       int *__restrict__ deg, unsigned long long *ghist)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    long long key = -1;
    if (v < n) {
        const int d = (int)((long long)off[v + 1] - (long long)off[v]);
        deg[v] = d;
        key = seg_key(vstart, G, v, d);
    }
    const unsigned int peers = __match_any_sync(0xffffffffu, key);
    if (v < n && lane == __ffs(peers) - 1)
        atomicAdd(&ghist[key], (unsigned long long)__popc(peers));
}

// rank[v] = start of its (graph, bucket) + arrival in it; order[rank] = v;
// rank_end[v] = the end of v's graph's ranks.  cursor = the exclusive scan of
// ghist, whose graph-major order places graph g's buckets at vstart[g].
__global__ void seg_rank_kernel(const int *__restrict__ deg, long long n,
                                const long long *__restrict__ vstart, long long G,
                                unsigned long long *cursor, int *__restrict__ rank,
                                int *__restrict__ order, int *__restrict__ rank_end)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    long long key = -1;
    if (v < n) {
        const long long g = seg_of(vstart, G, v);
        const int d = deg[v];
        key = g * kSegBuckets + degree_bucket<kSegBuckets>(d);
        rank_end[v] = (int)vstart[g + 1];    // the graph's ranks end where its vertices do
    }
    const unsigned int peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    unsigned long long at = 0;
    if (v < n && lane == leader) at = atomicAdd(&cursor[key], (unsigned long long)__popc(peers));
    at = __shfl_sync(0xffffffffu, at, leader);
    if (v < n) {
        const int r = (int)(at + __popc(peers & ((1u << lane) - 1u)));
        rank[v] = r;
        order[r] = (int)v;
    }
}

// Rows consumed at merge-path diagonal `diag` of the merge of the row-end
// offsets off[1..n] with the entry indices 0..nnz-1 (Merrill & Garland,
// "Merge-based parallel sparse matrix-vector multiplication", SC'16).
template <typename OffT>
__device__ __forceinline__ long long mp_rows(const OffT *__restrict__ off,
                                             long long n, long long nnz,
                                             long long diag)
{
    long long lo = diag - nnz > 0 ? diag - nnz : 0;
    long long hi = diag < n ? diag : n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if ((long long)off[mid + 1] <= diag - mid - 1) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Shared state of one merge-path tile: rows r0..r1 (offsets staged from
// off[r0]) and entries e0..e1 (adjacency staged).
struct TileSmem {
    long long off[kPrepTile + 2];
    int ind[kPrepTile];
    long long r0, e0, r1, e1;
};

// Merge-path coordinates of every tile boundary, all tiles at once (one
// thread per boundary), so the tile kernels start without a dependent search.
template <typename OffT>
__global__ void tile_bounds_kernel(const OffT *__restrict__ off, long long n,
                                   long long nnz, long long n_tiles,
                                   long long *__restrict__ trow, int *__restrict__ fcnt)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    long long d = t * kPrepTile;
    if (d > n + nnz) d = n + nnz;
    const long long r = mp_rows(off, n, nnz, d);
    trow[t] = r;
    // the row holding this boundary may be split between two tiles, which
    // then add their forward counts to fcnt[r]
    if (r < n) fcnt[r] = 0;
}

template <typename OffT>
__device__ void tile_stage(TileSmem &s, const OffT *__restrict__ off,
                           const int *__restrict__ ind, long long n,
                           long long nnz, const long long *__restrict__ trow)
{
    long long d0 = (long long)blockIdx.x * kPrepTile;
    long long d1 = d0 + kPrepTile;
    if (d1 > n + nnz) d1 = n + nnz;
    const long long r0 = trow[blockIdx.x], r1 = trow[blockIdx.x + 1];
    const long long e0 = d0 - r0, e1 = d1 - r1;
    if (threadIdx.x == 0) {
        s.r0 = r0; s.e0 = e0; s.r1 = r1; s.e1 = e1;
    }
    // off[r0 .. r1+1], clamped to off[n]
    for (long long k = threadIdx.x; k <= r1 - r0 + 1; k += blockDim.x) {
        long long r = r0 + k;
        s.off[k] = (long long)off[r <= n ? r : n];
    }
    for (long long k = threadIdx.x; k < e1 - e0; k += blockDim.x)
        s.ind[k] = ind[e0 + k];
    __syncthreads();
}

// Local merge-path start of this thread inside the staged tile.
__device__ __forceinline__ void tile_thread_start(const TileSmem &s,
                                                  long long &li, long long &lj)
{
    const long long rows = s.r1 - s.r0, ents = s.e1 - s.e0;
    long long ld = (long long)threadIdx.x * kPrepItemsPerThread;
    if (ld > rows + ents) ld = rows + ents;
    long long lo = ld - ents > 0 ? ld - ents : 0;
    long long hi = ld < rows ? ld : rows;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (s.off[mid + 1] - s.e0 <= ld - mid - 1) lo = mid + 1; else hi = mid;
    }
    li = lo;
    lj = ld - lo;
}

// This thread's items of the staged tile, classified from shared memory
// only: row ends and entries (with the entry's neighbour id and its row's
// degree), so that the degree gathers of all entries can be issued at once.
struct ThreadItems {
    unsigned int entry_mask;                 // bit k: item k is an entry
    unsigned int rowend_mask;                // bit k: item k ends a row
    int x[kPrepItemsPerThread];              // neighbour id (entries)
    int da[kPrepItemsPerThread];             // degree of the entry's row
    int rowloc[kPrepItemsPerThread];         // local row index of the item
};

__device__ __forceinline__ void tile_classify(const TileSmem &s, ThreadItems &it)
{
    long long li, lj;
    tile_thread_start(s, li, lj);
    const long long rows = s.r1 - s.r0, ents = s.e1 - s.e0;
    it.entry_mask = it.rowend_mask = 0;
#pragma unroll
    for (int k = 0; k < kPrepItemsPerThread; ++k) {
        it.x[k] = 0;
        it.da[k] = 0;
        it.rowloc[k] = (int)li;
        if (li + lj < rows + ents) {
            if (li < rows && lj >= s.off[li + 1] - s.e0) {
                it.rowend_mask |= 1u << k;
                ++li;
            } else {
                it.entry_mask |= 1u << k;
                it.x[k] = s.ind[lj];
                it.da[k] = (int)(s.off[li + 1] - s.off[li]);
                ++lj;
            }
        }
    }
}

// Forward flags of the thread's entries (bit k for item k), with every
// key gather issued before any flag is computed (skewed graphs, whose
// neighbour keys are scattered over memory).  Degree keys (RANK = false):
// an entry is forward when (deg x, x) > (deg row, row).  Rank keys: when
// rank x > rank row; the gathered ranks are returned in rx for the fill.
template <bool RANK>
__device__ __forceinline__ unsigned int forward_flags(const TileSmem &s, const ThreadItems &it,
                                                      const int *__restrict__ key, long long n,
                                                      unsigned int *status,
                                                      int (&rx)[kPrepItemsPerThread])
{
    unsigned int flags = 0;
    int ra[kPrepItemsPerThread];
#pragma unroll
    for (int k = 0; k < kPrepItemsPerThread; ++k) {
        const bool ok = ((it.entry_mask >> k) & 1u) &&
                        (unsigned long long)(long long)it.x[k] < (unsigned long long)n;
        rx[k] = ok ? key[it.x[k]] : 0;
        ra[k] = (RANK && ok) ? key[s.r0 + it.rowloc[k]] : 0;
    }
#pragma unroll
    for (int k = 0; k < kPrepItemsPerThread; ++k) {
        if (!((it.entry_mask >> k) & 1u)) continue;
        if ((unsigned long long)(long long)it.x[k] >= (unsigned long long)n) {
            atomicOr(status, kErrIndexRange);
            continue;
        }
        const bool fwd = RANK ? rx[k] > ra[k]
                              : rank_above(rx[k], it.x[k], it.da[k], (int)(s.r0 + it.rowloc[k]));
        if (fwd) flags |= 1u << k;
    }
    return flags;
}

// Single-pass forward-list build: every row's forward entries go to its own
// CSR segment, find[off[v] .. off[v] + d+(v)), and d+(v) to fcnt[v].  A
// tile places the rows it holds whole at positions from its block scan and
// stores their counts; a row split across tiles (at most the first and the
// last row of a tile) takes its positions for this tile's part from an
// atomic add on fcnt[v] (zeroed by tile_bounds_kernel), so the parts of such
// a row land in tile order of arrival.  Members keep the row's id order
// except across those parts; sort_lists_kernel restores the order wherever
// a consumer needs it.  With rank keys the lists hold the members' ranks.
template <typename OffT, bool RANK>
__global__ void __launch_bounds__(kPrepThreads, RANK ? 5 : 6)     // measured best per key type
tile_place_kernel(const OffT *__restrict__ off, const int *__restrict__ ind,
                  const int *__restrict__ key, long long n, long long nnz,
                  const long long *__restrict__ trow, int *__restrict__ fcnt,
                  int *__restrict__ find, unsigned int *status)
{
    __shared__ TileSmem s;
    __shared__ int warp_sum[kPrepThreads / 32];
    __shared__ int s_carry[2];
    tile_stage(s, off, ind, n, nnz, trow);
    ThreadItems it;
    tile_classify(s, it);
    int rx[kPrepItemsPerThread];
    const unsigned int flags = forward_flags<RANK>(s, it, key, n, status, rx);
    const int cnt = __popc(flags);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) warp_sum[warp] = incl;
    const long long r0 = s.r0;
    const int rows = (int)(s.r1 - s.r0);
    const bool first_split = s.off[0] < s.e0;              // row r0 began in an earlier tile
    const bool last_split = s.e1 > s.off[rows];            // row r1 goes on in a later tile
    const int nloc = rows + (last_split ? 1 : 0);          // rows with items in this tile
    __syncthreads();                                       // s.off is free from here on
    int base = 0, total = 0;
    for (int i = 0; i < kPrepThreads / 32; ++i) {
        if (i < warp) base += warp_sum[i];
        total += warp_sum[i];
    }
    const int pos0 = base + incl - cnt;                    // this thread's first local slot
    int *rowbase = reinterpret_cast<int *>(s.off);         // local slot of each row's first member
    if (threadIdx.x == 0) {
        rowbase[0] = 0;
        rowbase[nloc] = total;
    }
    int p = pos0;
#pragma unroll
    for (int k = 0; k < kPrepItemsPerThread; ++k) {
        if ((it.rowend_mask >> k) & 1u) rowbase[it.rowloc[k] + 1] = p;
        else if ((flags >> k) & 1u) ++p;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_carry[0] = s_carry[1] = 0;
        if (nloc == 1 && (first_split || last_split)) {
            s_carry[0] = atomicAdd(&fcnt[r0], rowbase[1] - rowbase[0]);
        } else if (nloc > 1) {
            if (first_split) s_carry[0] = atomicAdd(&fcnt[r0], rowbase[1] - rowbase[0]);
            if (last_split)
                s_carry[1] = atomicAdd(&fcnt[r0 + nloc - 1], rowbase[nloc] - rowbase[nloc - 1]);
        }
    }
    for (int li = threadIdx.x; li < nloc; li += kPrepThreads) {
        const bool split = (li == 0 && first_split) || (li == nloc - 1 && last_split);
        if (!split) fcnt[r0 + li] = rowbase[li + 1] - rowbase[li];
    }
    __syncthreads();
    p = pos0;
#pragma unroll
    for (int k = 0; k < kPrepItemsPerThread; ++k) {
        if (!((it.rowend_mask >> k) & 1u) && ((flags >> k) & 1u)) {
            const int li = it.rowloc[k];
            const int carry = li == 0 ? s_carry[0] : (li == nloc - 1 ? s_carry[1] : 0);
            find[(long long)off[r0 + li] + carry + (p - rowbase[li])] = RANK ? rx[k] : it.x[k];
            ++p;
        }
    }
}

// Sort one list of len <= 32*E ascending with the whole warp, in registers:
// lane l holds elements l*E .. l*E+E-1 (padded with +infinity), bitonic
// network with comparator distance j done inside a lane (j < E) or across
// lanes by shuffle (j >= E).
template <int E>
__device__ __forceinline__ void warp_sort_regs(int *list, int len, int lane)
{
    int v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane * E + e;
        v[e] = i < len ? list[i] : 0x7fffffff;
    }
#pragma unroll
    for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= E) {
                const int lj = j / E;
                const bool lower = (lane & lj) == 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const bool asc = k >= E ? (lane & (k / E)) == 0 : (e & k) == 0;
                    const int y = __shfl_xor_sync(0xffffffffu, v[e], lj);
                    v[e] = (lower == asc) ? min(v[e], y) : max(v[e], y);
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    if ((e & j) == 0) {
                        const bool asc = k >= E ? (lane & (k / E)) == 0 : (e & k) == 0;
                        const int a = v[e], b = v[e + j];
                        v[e] = asc ? min(a, b) : max(a, b);
                        v[e + j] = asc ? max(a, b) : min(a, b);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane * E + e;
        if (i < len) list[i] = v[e];
    }
}

// Lists longer than kSortRegMax, sorted in place in global memory by the
// warp: a bitonic sorter with ascending comparators only (the first step of
// every merge size k compares i with its mirror in the k-block, the later
// steps compare i with i + j).  Positions >= len hold +infinity implicitly:
// a comparator that touches one never moves anything, so it is skipped.
__device__ void warp_sort_global(int *list, int len, int lane)
{
    const int lp = ceil_log2(len);
    const int half = 1 << (lp - 1);
    for (int lk = 1; lk <= lp; ++lk) {
        const int k = 1 << lk;
        for (int lj = lk - 1; lj >= 0; --lj) {
            const int j = 1 << lj;
            const bool mirror = lj == lk - 1;
            for (int t = lane; t < half; t += 32) {
                const int lo = ((t >> lj) << (lj + 1)) | (t & (j - 1));
                const int hi = mirror ? ((lo & ~(k - 1)) + (k - 1) - (lo & (k - 1))) : lo + j;
                if (hi < len) {
                    const int a = list[lo], b = list[hi];
                    if (a > b) { list[lo] = b; list[hi] = a; }
                }
            }
            __syncwarp();
        }
    }
}

// One list of len >= 2 sorted by the whole warp: in registers up to
// kSortRegMax, in place in global memory beyond.
__device__ __forceinline__ void warp_sort_list(int *list, int len, int lane)
{
    if (len <= 32) warp_sort_regs<1>(list, len, lane);
    else if (len <= 64) warp_sort_regs<2>(list, len, lane);
    else if (len <= 128) warp_sort_regs<4>(list, len, lane);
    else if (len <= 256) warp_sort_regs<8>(list, len, lane);
    else if (len <= 512) warp_sort_regs<16>(list, len, lane);
    else if (len <= kSortRegMax) warp_sort_regs<32>(list, len, lane);
    else warp_sort_global(list, len, lane);
}

// Sort every forward list longer than min_len ascending (rank labels:
// min_len = min(cap, 31), cap = 4 * group the largest warp-kernel apex list).
// The lists read in order are the block-kernel apexes' (longer than cap) and
// the long partners' (32 or more); shorter lists are only ever read whole (as
// warp-kernel apexes, whose tables do not care about order, or as short
// partners, whose members are each checked against the apex rank).
// One warp per 32 consecutive rows, one list at a time (warp_sort_list).
// Groups come from a dynamic queue, so the few groups holding several long
// lists do not set the kernel's length.
template <typename OffT>
__global__ void __launch_bounds__(kSortThreads, 4)
sort_lists_kernel(const OffT *__restrict__ off, const int *__restrict__ fcnt, long long n,
                  int *__restrict__ find, Counters *ctr, int min_len)
{
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned long long grp = 0;
        if (lane == 0) grp = atomicAdd(&ctr->sort_groups, 1ull);
        const long long v0 = (long long)__shfl_sync(0xffffffffu, grp, 0) * 32;
        if (v0 >= n) break;
        const long long v = v0 + lane;
        long long b = 0, e = 0;
        if (v < n) { b = (long long)off[v]; e = b + fcnt[v]; }
        const long long ln = e - b;
        unsigned int todo = __ballot_sync(0xffffffffu, ln > min_len);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const long long lb = __shfl_sync(0xffffffffu, b, src);
            const int len = (int)__shfl_sync(0xffffffffu, ln, src);
            warp_sort_list(find + lb, len, lane);
            __syncwarp();
        }
    }
}

// Work items of the two count kernels, written by the row that owns them so
// that neither kernel starts an item with a search:
//   * block-kernel items: a row whose forward list exceeds the warp kernel's
//     table gets ceil(deg / big_chunk) items (row, chunk), at positions taken
//     from one atomic counter, one add per group of converged lanes (their
//     order does not matter; a batch posts about a million such rows);
//   * warp-kernel items: item k covers entries [k*item_len, (k+1)*item_len);
//     the row holding entry k*item_len records itself as the item's first row.
template <typename OffT>
__device__ __forceinline__ void post_row_items(long long v, long long b, long long e, int d,
                                               int fdeg, int small_cap, int big_chunk,
                                               int item_shift, Counters *ctr,
                                               int2 *__restrict__ bitem,
                                               long long *__restrict__ irow)
{
    if (fdeg > small_cap) {
        const int k = (int)div_up<long long>(d, big_chunk);
        // one atomic per group of converged lanes that post items
        auto grp = cg::coalesced_threads();
        const int incl = cg::inclusive_scan(grp, k);
        const int last = (int)grp.size() - 1;
        unsigned long long base = 0;
        if ((int)grp.thread_rank() == last)
            base = atomicAdd(&ctr->big_total, (unsigned long long)incl);
        base = grp.shfl(base, last);
        const unsigned long long at = base + (unsigned long long)(incl - k);
        for (int c = 0; c < k; ++c) bitem[at + c] = make_int2((int)v, c);
    }
    // items whose first entry lies in [b, e) (item_len = 2^item_shift)
    const long long mask = (1ll << item_shift) - 1;
    for (long long k = (b + mask) >> item_shift; (k << item_shift) < e; ++k) irow[k] = v;
}

// Rank labels: per-vertex record and work items (one thread per vertex).
template <typename OffT>
__global__ void vinfo_kernel(const OffT *__restrict__ off, const int *__restrict__ fcnt,
                             const int *__restrict__ deg, const int *__restrict__ rank,
                             long long n, int small_cap, int big_chunk, int item_shift,
                             VInfo *__restrict__ vinfo, Counters *ctr,
                             int2 *__restrict__ bitem, long long *__restrict__ irow)
{
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    VInfo r;
    r.fbeg = (long long)off[v];
    r.fdeg = fcnt[v];
    const int d = deg[v];
    r.key = rank[v];
    vinfo[v] = r;
    post_row_items<OffT>(v, r.fbeg, r.fbeg + d, d, r.fdeg, small_cap, big_chunk, item_shift, ctr,
                         bitem, irow);
}

// Vertex-id labels: the whole forward build in one pass.  Each row's entries
// are read in chunks by a group of GS lanes, which takes each neighbour's
// degree from the offsets, keeps the entries ordered above the row ((degree,
// id) order) and writes them, compacted by ballot, to the start of the row's
// own CSR segment -- so every list keeps the row's ascending id order and
// needs no sort.  Then the row's deg, fcnt, per-vertex record and work items
// are written.  Two launch forms:
//   * row_place_kernel: one group per row, its first lane writing the row's
//     records (small graphs: the most groups in flight);
//   * row_place_lane_kernel (below): a thread per row, from kRowPlaceThreadMin
//     rows on (large graphs).
template <int GS>
__device__ __forceinline__ int place_row(const int *__restrict__ ind, const void *offp,
                                         bool off32, long long n, long long v, long long b,
                                         int dv, int glane, int *__restrict__ find,
                                         unsigned int *status)
{
    auto off_at = [&](long long i) -> long long {
        return off32 ? (long long)static_cast<const int *>(offp)[i]
                     : static_cast<const long long *>(offp)[i];
    };
    auto grp = cg::tiled_partition<GS>(cg::this_thread_block());
    int wrote = 0;
    for (int k0 = 0; k0 < dv; k0 += GS) {
        const int k = k0 + glane;
        bool fwd = false;
        int x = 0;
        if (k < dv) {
            x = ind[b + k];
            if ((unsigned long long)(long long)x < (unsigned long long)n) {
                const int dx = (int)(off_at(x + 1) - off_at(x));
                fwd = dx > dv || (dx == dv && x > v);
            } else {
                atomicOr(status, kErrIndexRange);
            }
        }
        const unsigned int m = grp.ballot(fwd);
        if (fwd) find[b + wrote + __popc(m & ((1u << glane) - 1u))] = x;
        wrote += __popc(m);
    }
    return wrote;
}

template <typename OffT>
__device__ __forceinline__ void row_records(const OffT *off, long long v, long long b,
                                            long long e, int wrote, int small_cap,
                                            int big_chunk, int item_shift, int *__restrict__ deg,
                                            int *__restrict__ fcnt, VInfo *__restrict__ vinfo,
                                            Counters *ctr, int2 *__restrict__ bitem,
                                            long long *__restrict__ irow)
{
    const int d = (int)(e - b);
    deg[v] = d;
    fcnt[v] = wrote;
    VInfo r;
    r.fbeg = b;
    r.fdeg = wrote;
    r.key = d;
    vinfo[v] = r;
    post_row_items<OffT>(v, b, e, d, wrote, small_cap, big_chunk, item_shift, ctr, bitem, irow);
}

template <typename OffT, int GS>
__global__ void __launch_bounds__(256)
row_place_kernel(const OffT *__restrict__ off, const int *__restrict__ ind, long long n,
                 int *__restrict__ deg, int *__restrict__ fcnt, int *__restrict__ find,
                 VInfo *__restrict__ vinfo, int small_cap, int big_chunk, int item_shift,
                 Counters *ctr, int2 *__restrict__ bitem, long long *__restrict__ irow,
                 unsigned int *status)
{
    const long long v = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / GS;
    if (v >= n) return;                      // uniform across the group
    const int glane = (threadIdx.x & 31) % GS;
    const long long b = (long long)off[v], e = (long long)off[v + 1];
    const int wrote = place_row<GS>(ind, off, sizeof(OffT) == 4, n, v, b, (int)(e - b), glane,
                                    find, status);
    if (glane == 0)
        row_records<OffT>(off, v, b, e, wrote, small_cap, big_chunk, item_shift, deg, fcnt, vinfo,
                          ctr, bitem, irow);
}

// Thread-per-row form of the forward build for large graphs: each thread
// walks its own row serially, four entries at a time (the four id loads, then
// the eight offset loads, issued together), appending the entries ordered
// above the row to the start of the row's segment; rows longer than
// kLongRowMin are listed for long_row_place_kernel, a block per row, so that
// a hub holds up no warp.  On a 4 M-vertex mean-degree-12 graph it issues
// 105 M warp instructions where a 16-lane group per row (rows taken in turn
// by a warp's groups) issued 256 M, and takes 0.19 ms instead of 0.31; the
// offsets gather sets the pace.
template <typename OffT>
__global__ void __launch_bounds__(256)
row_place_lane_kernel(const OffT *__restrict__ off, const int *__restrict__ ind, long long n,
                      int *__restrict__ deg, int *__restrict__ fcnt, int *__restrict__ find,
                      VInfo *__restrict__ vinfo, int small_cap, int big_chunk, int item_shift,
                      Counters *ctr, int2 *__restrict__ bitem, long long *__restrict__ irow,
                      int *__restrict__ long_rows, unsigned int *status)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const long long b = (long long)off[v], e = (long long)off[v + 1];
    const int d = (int)(e - b);
    if (d > kLongRowMin) {
        const unsigned long long at = atomicAdd(&ctr->long_rows, 1ull);
        long_rows[at] = (int)v;
        return;
    }
    int wrote = 0;
    bool bad = false;
    auto keep = [&](int x, long long dx) {
        if (dx > d || (dx == d && x > v)) find[b + wrote++] = x;
    };
    int k = 0;
    for (; k + 4 <= d; k += 4) {
        int x[4];
        long long dx[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = ind[b + k + j];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool ok = (unsigned long long)(long long)x[j] < (unsigned long long)n;
            bad |= !ok;
            dx[j] = ok ? (long long)off[x[j] + 1] - (long long)off[x[j]] : -1;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (dx[j] >= 0) keep(x[j], dx[j]);
    }
    for (; k < d; ++k) {
        const int x = ind[b + k];
        if ((unsigned long long)(long long)x < (unsigned long long)n)
            keep(x, (long long)off[x + 1] - (long long)off[x]);
        else
            bad = true;
    }
    if (bad) atomicOr(status, kErrIndexRange);
    row_records<OffT>(off, v, b, e, wrote, small_cap, big_chunk, item_shift, deg, fcnt, vinfo, ctr,
                      bitem, irow);
}

// The rows row_place_lane_kernel handed on (longer than kLongRowMin), a block
// per row from a dynamic queue: the block's warps each take a contiguous
// slice of the row, count their forward entries, place them after the
// earlier slices' (a block scan of the counts), and the row's records follow.
template <typename OffT>
__global__ void __launch_bounds__(256)
long_row_place_kernel(const OffT *__restrict__ off, const int *__restrict__ ind, long long n,
                      int *__restrict__ deg, int *__restrict__ fcnt, int *__restrict__ find,
                      VInfo *__restrict__ vinfo, int small_cap, int big_chunk, int item_shift,
                      Counters *ctr, int2 *__restrict__ bitem, long long *__restrict__ irow,
                      const int *__restrict__ long_rows, unsigned int *status)
{
    __shared__ long long s_idx;
    __shared__ int s_cnt[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long total = (long long)ctr->long_rows;
    while (true) {
        if (threadIdx.x == 0) s_idx = (long long)atomicAdd(&ctr->long_next, 1ull);
        __syncthreads();
        const long long idx = s_idx;
        if (idx >= total) break;
        const long long v = long_rows[idx];
        const long long b = (long long)off[v], e = (long long)off[v + 1];
        const int dv = (int)(e - b);
        const int per = (dv + 7) / 8;
        const int k_lo = min(wid * per, dv), k_hi = min(k_lo + per, dv);
        // pass 1: forward entries of this warp's slice
        auto fwd_at = [&](int k, int &x) -> bool {
            x = ind[b + k];
            if ((unsigned long long)(long long)x >= (unsigned long long)n) {
                atomicOr(status, kErrIndexRange);
                return false;
            }
            const int dx = (int)((long long)off[x + 1] - (long long)off[x]);
            return dx > dv || (dx == dv && x > v);
        };
        int cnt = 0;
        for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
            const int k = k0 + lane;
            int x = 0;
            const bool f = k < k_hi && fwd_at(k, x);
            cnt += __popc(__ballot_sync(0xffffffffu, f));
        }
        if (lane == 0) s_cnt[wid] = cnt;
        __syncthreads();
        int base = 0, wrote = 0;
        for (int i = 0; i < 8; ++i) {
            if (i < wid) base += s_cnt[i];
            wrote += s_cnt[i];
        }
        // pass 2: place them, in row order
        for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
            const int k = k0 + lane;
            int x = 0;
            const bool f = k < k_hi && fwd_at(k, x);
            const unsigned int m = __ballot_sync(0xffffffffu, f);
            if (f) find[b + base + __popc(m & ((1u << lane) - 1u))] = x;
            base += __popc(m);
        }
        if (threadIdx.x == 0)
            row_records<OffT>(off, v, b, e, wrote, small_cap, big_chunk, item_shift, deg, fcnt,
                              vinfo, ctr, bitem, irow);
        __syncthreads();
    }
}

// ============================================================ intersection

// Shared-memory open-addressing table of one apex's forward list: int32 keys
// (-1 = empty), linear probing, and a 16-bit hit counter per slot packed two
// to a word.  A counter never exceeds the number of partners probed against
// one table (<= the entries of one work item < 65536), so the low half never
// carries into the high half.
struct ApexTable {
    int *keys;
    unsigned int *hits;
    int log2_slots;
    unsigned int mask;

    __device__ __forceinline__ void insert(int key) const
    {
        unsigned int slot = hash_slot(key, log2_slots);
        while (true) {
            int prev = atomicCAS(&keys[slot], -1, key);
            if (prev == -1) return;
            slot = (slot + 1) & mask;
        }
    }
    // Slot of key, or -1.  The first probe resolves almost every lookup at
    // the load factors used (<= 1/4); the loop only runs for collisions.
    __device__ __forceinline__ int find(int key) const
    {
        unsigned int slot = hash_slot(key, log2_slots);
        int k = keys[slot];
        if (k != key && k != -1) {
            do {
                slot = (slot + 1) & mask;
                k = keys[slot];
            } while (k != key && k != -1);
        }
        return k == key ? (int)slot : -1;
    }
    __device__ __forceinline__ void add_hit(int slot) const
    {
        atomicAdd(&hits[slot >> 1], 1u << ((slot & 1) << 4));
    }
    __device__ __forceinline__ unsigned int hit_pair(int word) const { return hits[word]; }
};

// Lanes [lo, hi) of a batch as a bit mask (0 <= lo < hi <= 32).
__device__ __forceinline__ unsigned int lane_range(int lo, int hi)
{
    return (0xffffffffu >> (32 - hi)) & (0xffffffffu << lo);
}

// Binary search of a sorted global forward list (block kernel, apexes whose
// forward list is larger than the shared table).
__device__ __forceinline__ int sorted_find(const int *__restrict__ list,
                                           int len, int key)
{
    int lo = 0, hi = len;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int v = list[mid];
        if (v < key) lo = mid + 1; else hi = mid;
    }
    return (lo < len && list[lo] == key) ? lo : -1;
}

// One stride of up to G adjacency entries of apex `a` (entries s..s+G-1 of
// N(a), clipped to `end`): select the partners whose edge belongs to `a` and
// probe every element of their forward lists into the apex's lookup.
//   * a partner with at least G forward neighbours is swept by the whole
//     group, G coalesced loads at a time, two in flight;
//   * the shorter lists are concatenated and swept G probes at a time, each
//     lane finding its partner by a shuffle binary search over the work
//     prefix (co-rank).
// TRIM (rank labels, lists of more than 16 members sorted ascending): an
// element ranked at or below the apex (key ka) cannot be in N+(a), so it is
// never looked up, and a long partner is swept from its end down to the
// first element at or below ka.  With TRIM the block-kernel apex (fa > cap)
// owns every edge to a lower-ranked neighbour -- probing only the part of
// its list ranked above the apex -- and an edge to a higher-ranked x only
// when x is a warp-kernel row (fx <= cap) with fx <= fa; every other edge
// keeps the longer-list rule, which is the warp kernel's rule, so each edge
// has exactly one owner.
// Partner credits: a long partner's hits are one warp reduction; a short
// partner's hits are the popcount of each batch's hit ballot over the lanes
// that batch gives it.
//   lookup(w) -> slot >= 0 on a hit, -1 on a miss (called with w > ka when TRIM)
//   on_hit(slot, w): credit of the third vertex
// Returns this lane's hit count (the apex credit).  G = 32: a whole warp.
template <int G, bool PER_VERTEX, bool TRIM, typename Grp, class Lookup, class OnHit>
__device__ __forceinline__ unsigned int
probe_stride(const Grp &grp, long long s, long long end, int a, int ka, int fa, int cap,
             const int *__restrict__ ind, const VInfo *__restrict__ vinfo,
             const int *__restrict__ find, long long n,
             unsigned long long *__restrict__ tacc, unsigned int *status,
             const Lookup &lookup, const OnHit &on_hit)
{
    const int lane = grp.thread_rank();
    const long long e = s + lane;
    bool partner = false;
    int x = 0, fx = 0;
    long long fbx = 0;
    if (e < end) {
        x = ind[e];
        if ((unsigned long long)(long long)x < (unsigned long long)n) {
            const VInfo ix = vinfo[x];
            fx = ix.fdeg;
            fbx = ix.fbeg;
            const bool fwd = rank_above(ix.key, x, ka, a);
            if (TRIM) partner = fx > 0 && (!fwd || (fx <= cap && fx <= fa));
            else partner = fx > 0 && (fwd ? fx <= fa : fx < fa);
        } else {
            atomicOr(status, kErrIndexRange);
        }
    }
    unsigned int hits = 0;

    // (1) long partners, one list at a time
    unsigned int longs = grp.ballot(partner && fx >= G);
    while (longs) {
        const int src = __ffs(longs) - 1;
        longs &= longs - 1;
        const int *list = find + grp.shfl(fbx, src);
        const int len = grp.shfl(fx, src);
        const int px = grp.shfl(x, src);
        unsigned int hx = 0;
        if (TRIM) {
            // windows of kTrimLoads * G elements from the end, all loads of a
            // window in flight together
            for (int top = len; top > 0; top -= kTrimLoads * G) {
                int w[kTrimLoads];
#pragma unroll
                for (int u = 0; u < kTrimLoads; ++u) {
                    const int j = top - (u + 1) * G + lane;
                    w[u] = j >= 0 ? list[j] : ka;
                }
#pragma unroll
                for (int u = 0; u < kTrimLoads; ++u) {
                    const int sl = w[u] > ka ? lookup(w[u]) : -1;
                    if (sl >= 0) {
                        ++hx;
                        if (PER_VERTEX) on_hit(sl, w[u]);
                    }
                }
                // sorted: once a loaded element is at or below ka, so is
                // every element before it (lanes past the list start load ka)
                if (grp.any(w[kTrimLoads - 1] <= ka)) break;
            }
        } else {
            int j = lane;
            for (; j + G < len; j += 2 * G) {
                const int w0 = list[j];
                const int w1 = list[j + G];
                const int s0 = lookup(w0);
                const int s1 = lookup(w1);
                if (s0 >= 0) {
                    ++hx;
                    if (PER_VERTEX) on_hit(s0, w0);
                }
                if (s1 >= 0) {
                    ++hx;
                    if (PER_VERTEX) on_hit(s1, w1);
                }
            }
            if (j < len) {
                const int w0 = list[j];
                const int s0 = lookup(w0);
                if (s0 >= 0) {
                    ++hx;
                    if (PER_VERTEX) on_hit(s0, w0);
                }
            }
        }
        if (PER_VERTEX) {
            const unsigned int hs = __reduce_add_sync(0xffffffffu, hx);
            if (lane == 0 && hs) atomicAdd(&tacc[px], (unsigned long long)hs);
        }
        hits += hx;
    }

    // (2) short partners, flattened
    const int work = (partner && fx < G) ? fx : 0;
    const int incl = cg::inclusive_scan(grp, work);
    const int total = grp.shfl(incl, G - 1);
    const int excl = incl - work;
    unsigned int mine = 0;
    for (int f0 = 0; f0 < total; f0 += G) {
        const int f = f0 + lane;
        // co-rank: lane i owns flattened index f iff excl_i <= f < incl_i
        int i = 0;
#pragma unroll
        for (int step = G / 2; step >= 1; step >>= 1) {
            const int v = grp.shfl(incl, i + step - 1);
            if (v <= f) i += step;
        }
        const long long fb_i = grp.shfl(fbx, i);
        const int ex_i = grp.shfl(excl, i);
        bool hit = false;
        if (f < total) {
            const int w = find[fb_i + (f - ex_i)];
            const int slot = (!TRIM || w > ka) ? lookup(w) : -1;
            if (slot >= 0) {
                hit = true;
                if (PER_VERTEX) on_hit(slot, w);
            }
        }
        hits += hit;
        if (PER_VERTEX) {
            const unsigned int hm = grp.ballot(hit);
            if (work > 0) {
                const int lo = max(excl - f0, 0), hi = min(incl - f0, G);
                if (lo < hi) mine += __popc(hm & lane_range(lo, hi));
            }
        }
    }
    if (PER_VERTEX && mine) atomicAdd(&tacc[x], (unsigned long long)mine);
    return hits;
}

// Label of a forward-list member -> vertex id (rank labels map through
// order[]; vertex-id labels are the id).
__device__ __forceinline__ int label_vertex(const int *__restrict__ order, int w)
{
    return order ? order[w] : w;
}

// Credit every third vertex w hit in this table (once per (apex, w));
// threads [t0, t0 + step) cover the table.
__device__ __forceinline__ void flush_hits(const ApexTable &tab, int tsize, int t0, int step,
                                           unsigned long long *__restrict__ tacc,
                                           const int *__restrict__ order)
{
    for (int wd = t0; wd < (tsize >> 1); wd += step) {
        const unsigned int pair = tab.hit_pair(wd);
        if (pair) {
            const unsigned int lo = pair & 0xffffu, hi = pair >> 16;
            if (lo) atomicAdd(&tacc[label_vertex(order, tab.keys[2 * wd])], (unsigned long long)lo);
            if (hi) atomicAdd(&tacc[label_vertex(order, tab.keys[2 * wd + 1])],
                              (unsigned long long)hi);
        }
    }
}

// Shuffle co-rank: the lane i whose [incl_i - w_i, incl_i) holds f (incl is
// this lane's inclusive prefix of a per-lane count; lanes with count 0 are
// never returned for f < total).
__device__ __forceinline__ int warp_corank(int incl, int f)
{
    int i = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, incl, i + step - 1);
        if (v <= f) i += step;
    }
    return i;
}

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Slot of key in a table region [toff, toff + 2^lg), or -1.
__device__ __forceinline__ int region_find(const int *keys, int toff, int lg, int key)
{
    const unsigned int mask = (1u << lg) - 1u;
    unsigned int s = hash_slot(key, lg);
    int k = keys[toff + s];
    if (k != key && k != -1) {
        do {
            s = (s + 1) & mask;
            k = keys[toff + s];
        } while (k != key && k != -1);
    }
    return k == key ? toff + (int)s : -1;
}

__device__ __forceinline__ void region_insert(int *keys, int toff, int lg, int key)
{
    const unsigned int mask = (1u << lg) - 1u;
    unsigned int s = hash_slot(key, lg);
    while (atomicCAS(&keys[toff + s], -1, key) != -1) s = (s + 1) & mask;
}

// Warp-per-item kernel for apexes with short forward lists (0 < d+ <=
// small_cap).  A work item is a range of `item_len` adjacency entries taken
// from a dynamic queue; the warp handles all rows of the item together,
// up to 32 rows at a time, with warp-uniform control flow:
//   1. one lane per row loads the row's segment and record; each active row
//      gets its own region (2^ceil(log2(m d+)) slots, m = region_mult: load
//      factor <= 1/2 for low-degree graphs, <= 1/4 otherwise) of
//      the warp's shared table, placed by a prefix scan (rows that do not fit
//      wait for the next batch);
//   2. the rows' forward lists are inserted as one flattened stream;
//   3. the rows' entries are scanned 32 at a time for partners, which are
//      appended to a per-warp queue in shared memory (list start, length,
//      owning region); every 32 queued partners -- and the rest at the end
//      of the batch -- are probed as one flattened stream into their apexes'
//      regions (shuffle co-rank over the work prefix), so probe passes run
//      full rather than once per entry chunk;
//   4. a partner lane popcounts the hit ballot over its probe range and
//      credits itself; apex credits collect in a shared per-row sum, and the
//      per-slot 16-bit hit counters credit the third vertices, both flushed
//      once per batch.
// List positions are 32-bit when the offsets are (every position < 2^31).
template <bool PER_VERTEX, typename OffT>
__global__ void __launch_bounds__(kRowThreads, kRowMinBlocks)
count_rows_kernel(const OffT *__restrict__ off, const int *__restrict__ ind,
                  long long n, long long nnz, const VInfo *__restrict__ vinfo,
                  const int *__restrict__ find,
                  unsigned long long *__restrict__ tacc, Counters *ctr,
                  unsigned int *status, const long long *__restrict__ irow,
                  long long n_items, int item_len, int small_cap, int region_mult,
                  const int *__restrict__ order)
{
    constexpr int kWarps = kRowThreads / 32;
    constexpr int kQueue = 64;                 // partner records per warp (32 + one chunk)
    __shared__ int s_keys[kWarps][kRowSlots];
    __shared__ unsigned int s_hits[kWarps][PER_VERTEX ? kRowSlots / 2 : 1];
    using Pos = typename std::conditional<sizeof(OffT) == 4, int, long long>::type;
    __shared__ Pos s_qfb[kWarps][kQueue];
    __shared__ int s_qx[kWarps][kQueue], s_qfx[kWarps][kQueue], s_qrd[kWarps][kQueue];
    __shared__ unsigned int s_apex[kWarps][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int *keys = s_keys[wid];
    unsigned int *hitw = s_hits[wid];
    Pos *qfb = s_qfb[wid];
    int *qx = s_qx[wid], *qfx = s_qfx[wid], *qrd = s_qrd[wid];
    unsigned int *apex_sum = s_apex[wid];
    apex_sum[lane] = 0;
    __syncwarp();
    unsigned long long tri_local = 0;

    // Probe the partner lists of queue records [0, k) (k <= 32) into their
    // apexes' regions as one flattened stream; credits: the partner per lane,
    // the apex through its batch row's shared sum.
    auto probe_queue = [&](int k) {
        int x = 0, fx = 0, rdp = 0;
        Pos fb = 0;
        if (lane < k) {
            x = qx[lane];
            fx = qfx[lane];
            fb = qfb[lane];
            rdp = qrd[lane];
        }
        __syncwarp();
        const int pw = fx;
        const int pincl = warp_incl_scan(pw);
        const int ptot = __shfl_sync(0xffffffffu, pincl, 31);
        const int pexcl = pincl - pw;
        const Pos pbase = fb - pexcl;
        unsigned int mine = 0;
        for (int g0 = 0; g0 < ptot; g0 += 32) {
            const int g = g0 + lane;
            const int pp = warp_corank(pincl, g);
            const Pos fb_p = __shfl_sync(0xffffffffu, pbase, pp);
            const int rd_p = __shfl_sync(0xffffffffu, rdp, pp);
            bool hit = false;
            if (g < ptot) {
                const int slot = region_find(keys, rd_p & 0xffff, (rd_p >> 16) & 0xff,
                                             find[fb_p + g]);
                if (slot >= 0) {
                    hit = true;
                    if (PER_VERTEX) atomicAdd(&hitw[slot >> 1], 1u << ((slot & 1) << 4));
                }
            }
            const unsigned int hm = __ballot_sync(0xffffffffu, hit);
            if (pw > 0) {
                const int lo = max(pexcl - g0, 0), hi = min(pincl - g0, 32);
                if (lo < hi) mine += __popc(hm & lane_range(lo, hi));
            }
        }
        if (PER_VERTEX && mine) {
            atomicAdd(&tacc[x], (unsigned long long)mine);
            atomicAdd(&apex_sum[(rdp >> 24) & 31], mine);
        }
        tri_local += mine;
    };

    while (true) {
        long long item = 0;
        if (lane == 0) item = (long long)atomicAdd(&ctr->row_items, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items) break;
        const long long e0 = item * item_len;
        const long long e1 = (e0 + item_len < nnz) ? e0 + item_len : nnz;
        long long ra = irow[item];
        while (true) {
            // ---- 1. rows of this batch (lane = row ra + lane)
            const long long r = ra + lane;
            const bool exists = r < n;
            const long long rb = exists ? (long long)off[r] : nnz;
            const long long re = exists ? (long long)off[r + 1] : nnz;
            const bool in_item = exists && rb < e1;
            const long long s0 = rb > e0 ? rb : e0;
            const long long s1 = re < e1 ? re : e1;
            const int len = (in_item && s1 > s0) ? (int)(s1 - s0) : 0;
            VInfo vi{0, 0, 0};
            if (len > 0) vi = vinfo[r];
            bool act = len > 0 && vi.fdeg > 0 && vi.fdeg <= small_cap;
            const int lg = act ? max(ceil_log2((long long)region_mult * vi.fdeg), 2) : 0;
            const int ts = act ? (1 << lg) : 0;
            const int tincl = warp_incl_scan(ts);
            const int toff = tincl - ts;
            // region: offset | log2(size) << 16 | batch row << 24
            const int rdesc = toff | (lg << 16) | (lane << 24);
            const bool take = in_item && tincl <= kRowSlots;
            const unsigned int tmask = __ballot_sync(0xffffffffu, take);
            const int nrows = __popc(tmask);          // a prefix of the lanes
            if (nrows == 0) break;                    // row ra starts at or after e1
            act = act && take;
            const int total_slots = (int)__reduce_max_sync(0xffffffffu, act ? (unsigned)tincl : 0u);
            if (total_slots > 0) {
                for (int k = lane; k < total_slots; k += 32) keys[k] = -1;
                if (PER_VERTEX)
                    for (int k = lane; k < (total_slots >> 1); k += 32) hitw[k] = 0;
                __syncwarp();
                // ---- 2. insert the forward lists of the active rows
                const int fw = act ? vi.fdeg : 0;
                const int fincl = warp_incl_scan(fw);
                const int ftot = __shfl_sync(0xffffffffu, fincl, 31);
                const int fexcl = fincl - fw;
                for (int f0 = 0; f0 < ftot; f0 += 32) {
                    const int f = f0 + lane;
                    const int i = warp_corank(fincl, f);
                    const Pos fb_i = __shfl_sync(0xffffffffu, (Pos)vi.fbeg - fexcl, i);
                    const int rd_i = __shfl_sync(0xffffffffu, rdesc, i);
                    if (f < ftot)
                        region_insert(keys, rd_i & 0xffff, (rd_i >> 16) & 0xff, find[fb_i + f]);
                }
                __syncwarp();
                // ---- 3. scan the active rows' entries for partners, probe
                const int lw = act ? len : 0;
                const int lincl = warp_incl_scan(lw);
                const int ltot = __shfl_sync(0xffffffffu, lincl, 31);
                const int lexcl = lincl - lw;
                int qn = 0;
                for (int c0 = 0; c0 < ltot; c0 += 32) {
                    const int f = c0 + lane;
                    const int i = warp_corank(lincl, f);
                    const Pos s0_i = __shfl_sync(0xffffffffu, (Pos)s0 - lexcl, i);
                    const int fa_i = __shfl_sync(0xffffffffu, vi.fdeg, i);
                    const int ka_i = __shfl_sync(0xffffffffu, vi.key, i);
                    const int rd_i = __shfl_sync(0xffffffffu, rdesc, i);
                    const int a = (int)(ra + i);
                    bool partner = false;
                    int x = 0, fx = 0;
                    Pos fbx = 0;
                    if (f < ltot) {
                        x = ind[s0_i + f];
                        if ((unsigned long long)(long long)x < (unsigned long long)n) {
                            const VInfo ix = vinfo[x];
                            fx = ix.fdeg;
                            fbx = (Pos)ix.fbeg;
                            const bool fwd = rank_above(ix.key, x, ka_i, a);
                            partner = fx > 0 && (fwd ? fx <= fa_i : fx < fa_i);
                        } else {
                            atomicOr(status, kErrIndexRange);
                        }
                    }
                    // queue this chunk's partners; probe 32 at a time
                    const unsigned int pm = __ballot_sync(0xffffffffu, partner);
                    if (partner) {
                        const int pos = qn + __popc(pm & ((1u << lane) - 1u));
                        qx[pos] = x;
                        qfx[pos] = fx;
                        qfb[pos] = fbx;
                        qrd[pos] = rd_i;
                    }
                    qn += __popc(pm);
                    __syncwarp();
                    if (qn >= 32) {
                        probe_queue(32);
                        const int rest = qn - 32;
                        if (lane < rest) {
                            qx[lane] = qx[32 + lane];
                            qfx[lane] = qfx[32 + lane];
                            qfb[lane] = qfb[32 + lane];
                            qrd[lane] = qrd[32 + lane];
                        }
                        __syncwarp();
                        qn = rest;
                    }
                }
                if (qn > 0) probe_queue(qn);
                __syncwarp();
                // ---- 4. third-vertex and apex credits
                if (PER_VERTEX) {
                    const unsigned int as = apex_sum[lane];
                    if (as) {
                        atomicAdd(&tacc[ra + lane], (unsigned long long)as);
                        apex_sum[lane] = 0;
                    }
                    for (int k = lane; k < (total_slots >> 1); k += 32) {
                        const unsigned int pair = hitw[k];
                        if (pair) {
                            const unsigned int lo = pair & 0xffffu, hi = pair >> 16;
                            if (lo) atomicAdd(&tacc[label_vertex(order, keys[2 * k])],
                                              (unsigned long long)lo);
                            if (hi) atomicAdd(&tacc[label_vertex(order, keys[2 * k + 1])],
                                              (unsigned long long)hi);
                        }
                    }
                }
                __syncwarp();
            }
            // ---- next batch: the row after the last taken one
            const long long last = ra + nrows - 1;
            const long long last_end = __shfl_sync(0xffffffffu, re, nrows - 1);
            if (last_end >= e1 || last + 1 >= n) break;
            ra = last + 1;
            if ((long long)off[ra + 1] == last_end) ra = row_of_entry(off, n, last_end);
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) tri_local += __shfl_down_sync(0xffffffffu, tri_local, d);
    if (lane == 0 && tri_local) atomicAdd(&ctr->tri_total, tri_local);
}

// Lane-per-row kernel for low-degree graphs with vertex-id labels, in place
// of count_rows_kernel.  It takes the same edges: every oriented edge u -> w
// (w in N+(u)) whose longer forward list has at most small_cap members and
// whose shorter one is not empty -- the edges whose apex count_rows_kernel
// would own -- and counts |N+(u) ∩ N+(w)| by merging the two lists, which are
// in ascending id order (the forward build keeps each row's order).  A lane
// owns a row u and all its edges, so the credits need no cross-lane work:
// u's in a register (one atomic per row), w's per edge, and each third vertex
// x in N+(u) in a per-lane 8-bit shared counter flushed once per (u, x)
// (a count is at most small_cap - 1 <= 127).  Warps take 32 rows at a time
// from a dynamic queue.  Trades the flattened warp machinery of
// count_rows_kernel (about 200 warp instructions per row on a mean-degree-12
// graph) for short serial merges when every list is short.
template <bool PER_VERTEX>
__global__ void __launch_bounds__(kRowThreads)
merge_rows_kernel(long long n, const VInfo *__restrict__ vinfo, const int *__restrict__ find,
                  unsigned long long *__restrict__ tacc, Counters *ctr, int small_cap)
{
    extern __shared__ unsigned char s_hit[];           // [small_cap][kRowThreads]
    const int lane = threadIdx.x & 31;
    unsigned char *hit = s_hit + threadIdx.x;
    unsigned long long tri_local = 0;
    while (true) {
        unsigned long long grp = 0;
        if (lane == 0) grp = atomicAdd(&ctr->row_items, 1ull);
        const long long u0 = (long long)__shfl_sync(0xffffffffu, grp, 0) * 32;
        if (u0 >= n) break;
        const long long u = u0 + lane;
        int fu = 0;
        long long fb = 0;
        if (u < n) {
            const VInfo vi = vinfo[u];
            fu = vi.fdeg;
            fb = vi.fbeg;
        }
        if (fu > small_cap) fu = 0;                 // the block kernel's apex
        const int *A = find + fb;
        if (PER_VERTEX)
            for (int i = 0; i < fu; ++i) hit[i * kRowThreads] = 0;
        unsigned int cu = 0;
        for (int j = 0; j < fu; ++j) {
            const int w = A[j];
            const VInfo vw = vinfo[w];
            const int fw = vw.fdeg;
            if (fw == 0 || fw > small_cap) continue;
            const int *B = find + vw.fbeg;
            int i = 0, k = 0;
            int a = A[0], b = B[0];
            unsigned int cw = 0;
            while (true) {
                if (a == b) {
                    ++cw;
                    if (PER_VERTEX) ++hit[i * kRowThreads];
                }
                const int ni = i + (a <= b), nk = k + (b <= a);
                if (ni >= fu || nk >= fw) break;
                a = A[ni];
                b = B[nk];
                i = ni;
                k = nk;
            }
            if (PER_VERTEX && cw) atomicAdd(&tacc[w], (unsigned long long)cw);
            cu += cw;
        }
        if (PER_VERTEX && cu) {
            atomicAdd(&tacc[u], (unsigned long long)cu);
            for (int i = 0; i < fu; ++i) {
                const unsigned int c = hit[i * kRowThreads];
                if (c) atomicAdd(&tacc[A[i]], (unsigned long long)c);
            }
        }
        tri_local += cu;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) tri_local += __shfl_down_sync(0xffffffffu, tri_local, d);
    if (lane == 0 && tri_local) atomicAdd(&ctr->tri_total, tri_local);
}

// Block-per-row kernel for apexes whose forward list exceeds small_cap.
// Vertex-id labels: the whole block shares one hash table of up to
// kBigTableSlots slots (load factor <= 1/8 up to kBigTableSlots/8 keys,
// <= 1/2 up to kBigHashMaxFdeg); beyond big_hash_max the apex list is
// binary-searched in global memory.
// Rank labels: N+(a) lies in the ranks above the apex, (ka, n).  When that
// range has at most kDirectRanks ranks, the block keeps one 16-bit counter
// per rank in it (0xffff for ranks outside N+(a)): a probe is one 2-byte
// load and a compare, a hit one packed shared atomic.  Up to 32*kBitWords
// ranks, the block marks the apex's list in a shared bitmap over the range
// -- one 8-byte load and one bit test per probe, no collisions.  Each 32-bit word of marks travels with the number of marks
// below it, so a hit at rank w has index (marks below its word) +
// popcount(lower bits of its word) in the sorted apex list, which indexes
// its 32-bit hit counter.  Larger ranges use the hash table or the binary
// search, with the rank keys.
// Within an item the warps take 32-entry strides from a shared counter, so
// uneven partner work does not idle the block at its barriers.
template <bool PER_VERTEX, typename OffT, bool RANK>
__global__ void __launch_bounds__(kBigThreads, kBigMinBlocks)
count_big_kernel(const OffT *__restrict__ off, const int *__restrict__ ind,
                 long long n, const VInfo *__restrict__ vinfo,
                 const int *__restrict__ find,
                 unsigned long long *__restrict__ tacc, Counters *ctr,
                 unsigned int *status, const int2 *__restrict__ bitem, int big_chunk,
                 int big_hash_max, int small_cap, const int *__restrict__ order,
                 const int *__restrict__ rank_end)
{
    extern __shared__ int smem[];
    int *keys = smem;
    unsigned int *hitw = reinterpret_cast<unsigned int *>(smem + kBigTableSlots);
    __shared__ long long s_item;
    __shared__ unsigned int s_cnt;
    __shared__ int s_next;
    __shared__ unsigned int s_wsum[kBigThreads / 32];
    auto block = cg::this_thread_block();
    auto warp = cg::tiled_partition<32>(block);
    const int lane = warp.thread_rank();
    const long long n_items = (long long)ctr->big_total;
    unsigned long long tri_local = 0;

    while (true) {
        if (threadIdx.x == 0) {
            s_item = (long long)atomicAdd(&ctr->big_items, 1ull);
            s_cnt = 0;
            s_next = 0;
        }
        __syncthreads();
        const long long item = s_item;
        if (item >= n_items) break;
        const int2 it = bitem[item];
        const long long a = it.x;
        const long long chunk = it.y;
        const long long rb = (long long)off[a] + chunk * big_chunk;
        long long re = rb + big_chunk;
        if (re > (long long)off[a + 1]) re = off[a + 1];
        const VInfo ia = vinfo[a];
        const int fa = ia.fdeg, ka = ia.key;
        const int *alist = find + ia.fbeg;
        unsigned int cnt = 0;
        auto next_stride = [&]() {
            int st = 0;
            if (lane == 0) st = atomicAdd(&s_next, 1);
            return rb + 32ll * warp.shfl(st, 0);
        };
        // N+(a) and every partner list lie in (ka, end): end = n, or with a
        // batch's graph-major ranks the end of the apex's own graph's ranks
        const long long range = RANK ? (rank_end ? (long long)rank_end[a] : n) - 1 - ka : n;
        if (RANK && range <= kDirectRanks) {
            // one 16-bit counter per rank above the apex; 0xffff marks a
            // rank outside N+(a), so the counter is also the membership test
            unsigned short *cnt16 = reinterpret_cast<unsigned short *>(smem);
            unsigned int *cnt32 = reinterpret_cast<unsigned int *>(smem);
            const int words = (int)((range + 1) >> 1);
            for (int k = threadIdx.x; k < words; k += kBigThreads) cnt32[k] = 0xffffffffu;
            __syncthreads();
            for (int k = threadIdx.x; k < fa; k += kBigThreads) cnt16[alist[k] - ka - 1] = 0;
            __syncthreads();
            auto lookup = [cnt16, ka](int w) -> int {
                const int p = w - ka - 1;
                return cnt16[p] != 0xffffu ? p : -1;
            };
            auto on_hit = [cnt32](int p, int) {
                atomicAdd(&cnt32[p >> 1], 1u << ((p & 1) << 4));
            };
            for (long long s = next_stride(); s < re; s = next_stride())
                cnt += probe_stride<32, PER_VERTEX, true>(warp, s, re, (int)a, ka, fa, small_cap,
                                                          ind, vinfo, find, n, tacc, status,
                                                          lookup, on_hit);
            __syncthreads();
            if (PER_VERTEX) {
                for (int k = threadIdx.x; k < fa; k += kBigThreads) {
                    const int w = alist[k];
                    const unsigned int c = cnt16[w - ka - 1];
                    if (c) atomicAdd(&tacc[order[w]], (unsigned long long)c);
                }
            }
        } else if (RANK && range <= 32ll * kBitWords && fa <= kBitKeys) {
            // word wd: .x = marks of ranks ka+1+32wd .. ka+32+32wd, .y = marks below
            uint2 *bw = reinterpret_cast<uint2 *>(smem);
            unsigned int *hitc = hitw;               // one 32-bit counter per apex element
            const int words = (int)((range + 31) >> 5);
            for (int k = threadIdx.x; k < words; k += kBigThreads) bw[k] = make_uint2(0u, 0u);
            if (PER_VERTEX)
                for (int k = threadIdx.x; k < fa; k += kBigThreads) hitc[k] = 0;
            __syncthreads();
            for (int k = threadIdx.x; k < fa; k += kBigThreads) {
                const unsigned int p = (unsigned int)(alist[k] - ka - 1);
                atomicOr(&bw[p >> 5].x, 1u << (p & 31u));
            }
            __syncthreads();
            if (PER_VERTEX) {
                constexpr int kPer = kBitWords / kBigThreads;
                const int w0 = threadIdx.x * kPer;
                unsigned int c = 0;
#pragma unroll
                for (int k = 0; k < kPer; ++k) c += (w0 + k < words) ? __popc(bw[w0 + k].x) : 0u;
                unsigned int incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const unsigned int o = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += o;
                }
                if (lane == 31) s_wsum[threadIdx.x >> 5] = incl;
                __syncthreads();
                unsigned int run = incl - c;
                for (int i = 0; i < (int)(threadIdx.x >> 5); ++i) run += s_wsum[i];
#pragma unroll
                for (int k = 0; k < kPer; ++k) {
                    if (w0 + k < words) {
                        bw[w0 + k].y = run;
                        run += __popc(bw[w0 + k].x);
                    }
                }
                __syncthreads();
            }
            auto lookup = [bw, ka](int w) -> int {
                const unsigned int p = (unsigned int)(w - ka - 1);
                const uint2 wd = bw[p >> 5];
                const unsigned int b = p & 31u;
                if (!((wd.x >> b) & 1u)) return -1;
                return PER_VERTEX ? (int)(wd.y + __popc(wd.x & ((1u << b) - 1u))) : 0;
            };
            auto on_hit = [hitc](int slot, int) { atomicAdd(&hitc[slot], 1u); };
            for (long long s = next_stride(); s < re; s = next_stride())
                cnt += probe_stride<32, PER_VERTEX, true>(warp, s, re, (int)a, ka, fa, small_cap,
                                                          ind, vinfo, find, n, tacc, status,
                                                          lookup, on_hit);
            __syncthreads();
            if (PER_VERTEX) {
                for (int k = threadIdx.x; k < fa; k += kBigThreads) {
                    const unsigned int c = hitc[k];
                    if (c) atomicAdd(&tacc[order[alist[k]]], (unsigned long long)c);
                }
            }
        } else if (fa <= big_hash_max) {
            const int log2t = min(max(ceil_log2(8 * (long long)fa), 6), kBigTableLog2);
            const int tsize = 1 << log2t;
            for (int k = threadIdx.x; k < tsize; k += kBigThreads) keys[k] = -1;
            if (PER_VERTEX)
                for (int k = threadIdx.x; k < (tsize >> 1); k += kBigThreads) hitw[k] = 0;
            __syncthreads();
            const ApexTable tab{keys, hitw, log2t, (unsigned int)(tsize - 1)};
            for (int k = threadIdx.x; k < fa; k += kBigThreads) tab.insert(alist[k]);
            __syncthreads();
            auto lookup = [tab](int w) { return tab.find(w); };
            auto on_hit = [tab](int slot, int) { tab.add_hit(slot); };
            for (long long s = next_stride(); s < re; s = next_stride())
                cnt += probe_stride<32, PER_VERTEX, RANK>(warp, s, re, (int)a, ka, fa, small_cap,
                                                          ind, vinfo, find, n, tacc, status,
                                                          lookup, on_hit);
            __syncthreads();
            if (PER_VERTEX) flush_hits(tab, tsize, threadIdx.x, kBigThreads, tacc, order);
        } else {
            auto lookup = [alist, fa](int w) { return sorted_find(alist, fa, w); };
            auto on_hit = [tacc, order](int, int w) {
                atomicAdd(&tacc[label_vertex(order, w)], 1ull);
            };
            for (long long s = next_stride(); s < re; s = next_stride())
                cnt += probe_stride<32, PER_VERTEX, RANK>(warp, s, re, (int)a, ka, fa, small_cap,
                                                          ind, vinfo, find, n, tacc, status,
                                                          lookup, on_hit);
        }
        const unsigned int wsum = cg::reduce(warp, cnt, cg::plus<unsigned int>());
        if (lane == 0 && wsum) atomicAdd(&s_cnt, wsum);
        __syncthreads();
        if (threadIdx.x == 0 && s_cnt) {
            if (PER_VERTEX) atomicAdd(&tacc[a], (unsigned long long)s_cnt);
            tri_local += s_cnt;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && tri_local) atomicAdd(&ctr->tri_total, tri_local);
}

// ================================================================ epilogue

__global__ void finalize_kernel(long long n,
                                const unsigned long long *__restrict__ tacc,
                                const int *__restrict__ deg,
                                long long *__restrict__ r,
                                long long *__restrict__ t,
                                double *__restrict__ lcc)
{
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const long long tv = (long long)tacc[v];
    if (r) r[v] = 2 * tv;
    if (t) t[v] = tv;
    if (lcc) {
        const long long d = deg[v];
        // one IEEE division of exactly converted integers (bit-identical
        // to the host formula)
        lcc[v] = (d < 2) ? 0.0 : __ddiv_rn((double)(2 * tv), (double)(d * (d - 1)));
    }
}

__global__ void global_kernel(const Counters *ctr, long long *global)
{
    const long long T = (long long)ctr->tri_total;
    global[0] = T;
    global[1] = 3 * T;
    global[2] = 6 * T;
}

// ================================================================== host

namespace {

// Host-side NVTX range around the launches of one pipeline phase (header-only
// NVTX 3: a no-op unless a profiler injects itself).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

int g_sm_count[64];
int g_rows_blocks[64][8];
int g_big_blocks[64][4];
int g_sort_blocks[64][2];
int g_merge_blocks[64][8];

int device_sm_count(int dev)
{
    if (dev < 0 || dev >= 64) return 148;
    if (!g_sm_count[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        g_sm_count[dev] = v > 0 ? v : 148;
    }
    return g_sm_count[dev];
}

template <typename K>
int occupancy_blocks(K kernel, int threads, size_t dyn_smem, int dev, int *cache)
{
    if (dev >= 0 && dev < 64 && *cache) return *cache;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * device_sm_count(dev);
    if (dev >= 0 && dev < 64) *cache = blocks;
    return blocks;
}

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

Plan make_plan(long long n, long long nnz, int off_bits, bool per_vertex)
{
    Plan p;
    p.n = n;
    p.nnz = nnz;
    p.off_bits = off_bits;
    p.n_tiles = div_up<long long>(n + nnz, kPrepTile);
    p.fwd_cap = nnz;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = align256(o + bytes); return at; };
    p.o_status = take(sizeof(unsigned int));
    p.o_counters = take(sizeof(Counters));
    p.o_hist = take(sizeof(unsigned long long) * (size_t)kRankBuckets);
    p.o_deg = take(sizeof(int) * (size_t)n);
    p.o_rank = take(sizeof(int) * (size_t)n);
    p.o_order = take(sizeof(int) * (size_t)n);
    p.o_fcnt = take(sizeof(int) * (size_t)n);
    p.o_vinfo = take(sizeof(VInfo) * (size_t)n);
    p.o_find = take(sizeof(int) * (size_t)(p.fwd_cap + 4));
    p.o_tacc = take(per_vertex ? sizeof(unsigned long long) * (size_t)n : 0);
    p.o_trow = take(sizeof(long long) * (size_t)(p.n_tiles + 1));
    p.o_irow = take(sizeof(long long) * (size_t)(div_up<long long>(nnz, kMinItemLen) + 1));
    // block-kernel items: at most one per row plus one per kMinBigChunk entries
    p.o_bitem = take(sizeof(int2) * (size_t)(n + div_up<long long>(nnz, kMinBigChunk) + 1));
    // rows longer than kLongRowMin, at most nnz / (kLongRowMin + 1) of them
    p.o_long = take(sizeof(int) * (size_t)(nnz / (kLongRowMin + 1) + 1));
    p.bytes = o;
    return p;
}

RowConfig pick_row_config(long long n, long long nnz)
{
    RowConfig c;
    const double avg = n > 0 ? (double)nnz / (double)n : 0.0;
    if (avg <= 24.0) {
        c.group = 8; c.item_len = 256; c.rank_labels = false; c.region_mult = 2;
    } else {
        c.group = 32; c.item_len = 512; c.rank_labels = true;
    }
    c.big_chunk = 2048;
    // small graphs: shorter warp items, so that there are enough to fill
    // every SM (an ER graph of 16,384 vertices counts 17% faster)
    if (nnz < (4ll << 20)) c.item_len = 128;
    // large graphs with vertex-id labels: per-row merges (a 4 M-vertex
    // mean-degree-12 graph's group kernel takes 0.87 ms instead of 0.97; a
    // 16 K-vertex ER graph's 0.062 instead of 0.037, hence the bound)
    c.merge_rows = !c.rank_labels && n >= kRowPlaceThreadMin;
    return c;
}

gtc_status apply_tuning(RowConfig &cfg, const gtc_tuning *tuning)
{
    if (!tuning) return GTC_OK;
    if (tuning->group) {
        if (tuning->group != 4 && tuning->group != 8 && tuning->group != 16 &&
            tuning->group != 32)
            return GTC_ERR_INVALID_ARGUMENT;
        cfg.group = tuning->group;
    }
    // item_len (a power of two) and big_chunk bound the 16-bit shared hit
    // counters: a counter collects at most one hit per adjacency entry of one
    // work item
    if (tuning->item_len < 0 || (tuning->item_len > 0 && tuning->item_len < kMinItemLen) ||
        tuning->item_len > kMaxItemLen || (tuning->item_len & (tuning->item_len - 1)) ||
        tuning->big_chunk < 0 || (tuning->big_chunk > 0 && tuning->big_chunk < kMinBigChunk) ||
        tuning->big_hash_max < 0 ||
        tuning->big_hash_max > kBigHashMaxFdeg || tuning->big_chunk > 32768 ||
        tuning->labels < 0 || tuning->labels > 2 ||
        (tuning->region != 0 && tuning->region != 2 && tuning->region != 4) ||
        tuning->rows < 0 || tuning->rows > 2 ||
        (tuning->rows == GTC_ROWS_MERGE && tuning->labels == GTC_LABELS_DEGREE_RANK))
        return GTC_ERR_INVALID_ARGUMENT;
    if (tuning->item_len) cfg.item_len = tuning->item_len;
    if (tuning->big_chunk) cfg.big_chunk = tuning->big_chunk;
    if (tuning->big_hash_max) cfg.big_hash_max = tuning->big_hash_max;
    if (tuning->labels == GTC_LABELS_VERTEX_ID) cfg.rank_labels = false;
    if (tuning->labels == GTC_LABELS_DEGREE_RANK) cfg.rank_labels = true;
    if (tuning->region) cfg.region_mult = tuning->region;
    if (tuning->rows == GTC_ROWS_HASH) cfg.merge_rows = false;
    if (tuning->rows == GTC_ROWS_MERGE) {
        cfg.merge_rows = true;
        cfg.rank_labels = false;
    }
    // the merge kernel needs id-ordered lists
    if (cfg.rank_labels) cfg.merge_rows = false;
    return GTC_OK;
}

int launches_per_count(const RowConfig &cfg, bool per_vertex, long long n)
{
    // vertex-id labels: row placement (and, from kRowPlaceThreadMin rows on,
    // the long-row placement); rank labels: degree histogram, rank scan,
    // rank, tile bounds, tile placement, list sort, vinfo.  Then the warp
    // kernel, the block kernel, the global count and, per vertex, finalize.
    const int build = cfg.rank_labels ? 7 : (n >= kRowPlaceThreadMin ? 2 : 1);
    return build + 3 + (per_vertex ? 1 : 0);
}

template <typename OffT>
gtc_status run_count(const OffT *off, const int *ind, long long n, long long nnz,
                     bool per_vertex, long long *r, long long *t, double *lcc,
                     long long *global, void *ws, size_t ws_bytes,
                     cudaStream_t stream, const RowConfig &cfg, CountTimings *timing,
                     const SegRanks *seg)
{
    const int off_bits = sizeof(OffT) * 8;
    Plan p = make_plan(n, nnz, off_bits, per_vertex);
    if (ws_bytes < p.bytes) return GTC_ERR_WORKSPACE_TOO_SMALL;
    char *base = static_cast<char *>(ws);
    unsigned int *status = reinterpret_cast<unsigned int *>(base + p.o_status);
    Counters *ctr = reinterpret_cast<Counters *>(base + p.o_counters);
    int *deg = reinterpret_cast<int *>(base + p.o_deg);
    int *fcnt = reinterpret_cast<int *>(base + p.o_fcnt);
    VInfo *vinfo = reinterpret_cast<VInfo *>(base + p.o_vinfo);
    int *find = reinterpret_cast<int *>(base + p.o_find);
    unsigned long long *tacc = reinterpret_cast<unsigned long long *>(base + p.o_tacc);
    long long *trow = reinterpret_cast<long long *>(base + p.o_trow);
    long long *irow = reinterpret_cast<long long *>(base + p.o_irow);
    int2 *bitem = reinterpret_cast<int2 *>(base + p.o_bitem);
    const bool rank_labels = cfg.rank_labels;
    unsigned long long *hist = reinterpret_cast<unsigned long long *>(base + p.o_hist);
    int *rank = reinterpret_cast<int *>(base + p.o_rank);
    int *order = reinterpret_cast<int *>(base + p.o_order);

    NvtxRange count_range("gtc_count");
    int dev = 0;
    cudaGetDevice(&dev);
    cudaError_t err;
    // status word, counters (and the rank histogram) lead the workspace
    err = cudaMemsetAsync(base, 0, rank_labels ? p.o_deg : p.o_hist, stream);
    if (err != cudaSuccess) return GTC_ERR_CUDA;
    if (per_vertex && n > 0) {
        err = cudaMemsetAsync(tacc, 0, sizeof(unsigned long long) * (size_t)n, stream);
        if (err != cudaSuccess) return GTC_ERR_CUDA;
    }
    if (n > 0) {
        const unsigned vb = (unsigned)div_up<long long>(n, 256);
        if (timing) cudaEventRecord(timing->ev[0], stream);
        nvtxRangePushA("gtc: forward lists");
        const int small_cap = 4 * cfg.group;   // <= kRowSlots / 8
        if (rank_labels) {
            if (seg && seg->num_graphs > 0) {
                const long long nb = seg->num_graphs * kSegBuckets;
                unsigned long long *gh = reinterpret_cast<unsigned long long *>(seg->ghist);
                err = cudaMemsetAsync(gh, 0, sizeof(long long) * (size_t)(nb + 1), stream);
                if (err != cudaSuccess) return GTC_ERR_CUDA;
                seg_degree_hist_kernel<OffT><<<vb, 256, 0, stream>>>(off, n, seg->vstart,
                                                                     seg->num_graphs, deg, gh);
                err = exclusive_scan_i64(seg->ghist, seg->ghist, nb, seg->scan_tmp, stream);
                if (err != cudaSuccess) return GTC_ERR_CUDA;
                seg_rank_kernel<<<vb, 256, 0, stream>>>(deg, n, seg->vstart, seg->num_graphs, gh,
                                                        rank, order, seg->rank_end);
            } else {
                const unsigned rb = (unsigned)div_up<long long>(n, kRankChunk);
                degree_hist_kernel<<<rb, kRankThreads, 0, stream>>>(off, off_bits, n, deg, hist);
                rank_scan_kernel<<<1, kRankScanThreads, 0, stream>>>(hist);
                rank_kernel<<<rb, kRankThreads, 0, stream>>>(deg, n, hist, rank, order);
            }
            tile_bounds_kernel<OffT><<<(unsigned)div_up<long long>(p.n_tiles + 1, 256), 256, 0,
                                       stream>>>(off, n, nnz, p.n_tiles, trow, fcnt);
            tile_place_kernel<OffT, true><<<(unsigned)p.n_tiles, kPrepThreads, 0, stream>>>(
                off, ind, rank, n, nnz, trow, fcnt, find, status);
            // rank order for the lists read in order (rows hold their members
            // in id order)
            long long sb = occupancy_blocks(sort_lists_kernel<OffT>, kSortThreads, 0, dev,
                                            &g_sort_blocks[dev & 63][off_bits == 32 ? 0 : 1]);
            const long long sneed = div_up<long long>(n, 32 * (kSortThreads / 32));
            if (sneed < sb) sb = sneed;
            sort_lists_kernel<OffT><<<(unsigned)sb, kSortThreads, 0, stream>>>(
                off, fcnt, n, find, ctr, min(4 * cfg.group, 31));
            vinfo_kernel<OffT><<<vb, 256, 0, stream>>>(off, fcnt, deg, rank, n, small_cap,
                                                       cfg.big_chunk, ceil_log2(cfg.item_len),
                                                       vinfo, ctr, bitem, irow);
        } else {
            // small graphs: a group of gs lanes (about the mean degree) per
            // row; from kRowPlaceThreadMin rows on a thread per row, the long
            // rows a block each
            const double mean = (double)nnz / (double)n;
            const int gs = mean <= 8.0 ? 8 : (mean <= 16.0 ? 16 : 32);
            const int ishift = ceil_log2(cfg.item_len);
            int *long_rows = reinterpret_cast<int *>(base + p.o_long);
            if (n >= kRowPlaceThreadMin) {
                row_place_lane_kernel<OffT><<<(unsigned)div_up<long long>(n, 256), 256, 0,
                                              stream>>>(off, ind, n, deg, fcnt, find, vinfo,
                                                        small_cap, cfg.big_chunk, ishift, ctr,
                                                        bitem, irow, long_rows, status);
                long_row_place_kernel<OffT><<<(unsigned)(device_sm_count(dev) * 4), 256, 0,
                                              stream>>>(off, ind, n, deg, fcnt, find, vinfo,
                                                        small_cap, cfg.big_chunk, ishift, ctr,
                                                        bitem, irow, long_rows, status);
            } else {
                const unsigned pb = (unsigned)div_up<long long>(n * gs, 256);
                auto place = [&](auto kern) {
                    kern<<<pb, 256, 0, stream>>>(off, ind, n, deg, fcnt, find, vinfo, small_cap,
                                                 cfg.big_chunk, ishift, ctr, bitem, irow, status);
                };
                if (gs == 8) place(row_place_kernel<OffT, 8>);
                else if (gs == 16) place(row_place_kernel<OffT, 16>);
                else place(row_place_kernel<OffT, 32>);
            }
        }
        nvtxRangePop();
        if (timing) cudaEventRecord(timing->ev[1], stream);
        const int *lorder = rank_labels ? order : nullptr;
        const int *rank_end = (rank_labels && seg && seg->num_graphs > 0) ? seg->rank_end : nullptr;
        if (nnz > 0) {
            const long long n_items = div_up<long long>(nnz, cfg.item_len);
            auto launch_rows = [&](auto kern) {
                int blocks = occupancy_blocks(kern, kRowThreads, 0, dev,
                                              &g_rows_blocks[dev & 63][per_vertex ? 1 : 0]);
                long long need = div_up<long long>(n_items, kRowThreads / 32);
                if (need < blocks) blocks = (int)need;
                kern<<<blocks, kRowThreads, 0, stream>>>(off, ind, n, nnz, vinfo, find, tacc, ctr,
                                                         status, irow, n_items, cfg.item_len,
                                                         small_cap, cfg.region_mult, lorder);
            };
            if (cfg.merge_rows && !rank_labels) {
                NvtxRange r("gtc: warp kernel");
                auto kern = per_vertex ? merge_rows_kernel<true> : merge_rows_kernel<false>;
                const size_t msmem = per_vertex ? (size_t)small_cap * kRowThreads : 0;
                int *cache = &g_merge_blocks[dev & 63][(per_vertex ? 4 : 0) +
                                                       (ceil_log2(cfg.group) & 3)];
                int blocks = occupancy_blocks(kern, kRowThreads, msmem, dev, cache);
                const long long need = div_up<long long>(n, kRowThreads);
                if (need < blocks) blocks = (int)need;
                kern<<<blocks, kRowThreads, msmem, stream>>>(n, vinfo, find, tacc, ctr, small_cap);
            } else {
                NvtxRange r("gtc: warp kernel");
                if (per_vertex) launch_rows(count_rows_kernel<true, OffT>);
                else launch_rows(count_rows_kernel<false, OffT>);
            }
            if (timing) cudaEventRecord(timing->ev[2], stream);
            const size_t big_smem = sizeof(int) * kBigTableSlots +
                                    sizeof(unsigned int) * (kBigTableSlots / 2);
            auto launch_big = [&](auto kern, int *cache) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem);
                int blocks = occupancy_blocks(kern, kBigThreads, big_smem, dev, cache);
                kern<<<blocks, kBigThreads, big_smem, stream>>>(off, ind, n, vinfo, find, tacc, ctr,
                                                                status, bitem, cfg.big_chunk,
                                                                cfg.big_hash_max, small_cap, lorder,
                                                                rank_end);
            };
            int *bc = g_big_blocks[dev & 63];
            NvtxRange r("gtc: block kernel");
            if (rank_labels) {
                if (per_vertex) launch_big(count_big_kernel<true, OffT, true>, &bc[3]);
                else launch_big(count_big_kernel<false, OffT, true>, &bc[2]);
            } else {
                if (per_vertex) launch_big(count_big_kernel<true, OffT, false>, &bc[1]);
                else launch_big(count_big_kernel<false, OffT, false>, &bc[0]);
            }
        } else if (timing) {
            cudaEventRecord(timing->ev[2], stream);
        }
        if (timing) cudaEventRecord(timing->ev[3], stream);
        if (per_vertex && (r || t || lcc))
            finalize_kernel<<<vb, 256, 0, stream>>>(n, tacc, deg, r, t, lcc);
    }
    if (global) global_kernel<<<1, 1, 0, stream>>>(ctr, global);
    if (timing) cudaEventRecord(timing->ev[4], stream);
    err = cudaGetLastError();
    return err == cudaSuccess ? GTC_OK : GTC_ERR_CUDA;
}

template gtc_status run_count<int>(const int *, const int *, long long, long long, bool,
                                   long long *, long long *, double *, long long *, void *,
                                   size_t, cudaStream_t, const RowConfig &, CountTimings *,
                                   const SegRanks *);
template gtc_status run_count<long long>(const long long *, const int *, long long, long long,
                                         bool, long long *, long long *, double *, long long *,
                                         void *, size_t, cudaStream_t, const RowConfig &,
                                         CountTimings *, const SegRanks *);

}  // namespace gtc
