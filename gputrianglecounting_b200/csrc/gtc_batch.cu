// gtc_batch.cu -- many independent graphs counted in one pipeline run.
//
// A batch is the disjoint union of its graphs: graph g owns the vertex range
// [vstart[g], vstart[g+1]) and the entry range [off[vstart[g]],
// off[vstart[g+1]]) of one concatenated CSR whose adjacency holds *local* ids
// (0 .. n_g-1).  The batch entry point turns local ids into union ids in one
// pass and runs the single-graph pipeline (persistent kernels pulling work
// items from device queues) once over the union; triangles never cross graphs,
// so every per-vertex value is exactly the one the graph gets alone.  With
// degree-rank labels the ranks are graph-major (each graph's vertices take the
// consecutive ranks vstart[g] ..), so an apex's forward list spans only its own
// graph's ranks and small graphs keep the block kernel's direct per-rank
// counters.  A final kernel sums t over each graph's vertex range into that
// graph's T.
// The reference has no batched form; its per-graph operator is kernelCall
// (src/clusteringCount.cu:415-467), which the one-launch-per-graph baseline
// calls once per graph.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "gtc_core.cuh"

namespace cg = cooperative_groups;

namespace gtc {
namespace {

constexpr int kChunk = 4096;     // entries (or vertices) per block

// estart[g] = off[vstart[g]] for g in [0, G]
__global__ void graph_entry_starts(const long long *__restrict__ off,
                                   const long long *__restrict__ vstart, long long G,
                                   long long *__restrict__ estart)
{
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g <= G) estart[g] = off[vstart[g]];
}

// Largest g in [0, G) with start[g] <= x (start non-decreasing, start[0] <= x).
__device__ __forceinline__ long long owner(const long long *__restrict__ start, long long G,
                                           long long x)
{
    long long lo = 0, hi = G;
    while (hi - lo > 1) {
        long long mid = (lo + hi) >> 1;
        if (start[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// ind_g[e] = ind[e] + vstart[graph of e]; a block covers kChunk entries, each
// thread four consecutive ones at a time (one 16-byte load and store when
// both arrays are 16-byte aligned), walking forward from the block's first
// graph with the current graph's bounds in registers (2.8 TB/s with one
// entry per thread and the bounds reloaded per entry; 5 ms instead of 9 on
// the 3.1 G-entry batch).  A local id outside its graph's [0, n_g) becomes
// -1, which the counting kernels flag (kErrIndexRange) and skip instead of
// crediting another graph's vertex.
template <bool VEC>
__global__ void globalize_kernel(const long long *__restrict__ estart,
                                 const long long *__restrict__ vstart, long long G,
                                 const int *__restrict__ ind, int *__restrict__ ind_g,
                                 long long nnz)
{
    __shared__ long long s_g0;
    const long long e_begin = (long long)blockIdx.x * kChunk;
    if (threadIdx.x == 0) s_g0 = owner(estart, G, e_begin);
    __syncthreads();
    long long g = s_g0;
    long long g_end = g + 1 < G ? estart[g + 1] : nnz;      // first entry past graph g
    long long v0 = vstart[g], nv = vstart[g + 1] - v0;
    const long long e_stop = e_begin + kChunk < nnz ? e_begin + kChunk : nnz;
    for (long long e4 = e_begin + 4ll * threadIdx.x; e4 < e_stop; e4 += 4ll * blockDim.x) {
        int x[4];
        if (VEC && e4 + 4 <= e_stop) {
            const int4 q = *reinterpret_cast<const int4 *>(ind + e4);
            x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) x[j] = e4 + j < e_stop ? ind[e4 + j] : 0;
        }
        int y[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            while (e4 + j >= g_end && g + 1 < G) {
                ++g;
                g_end = g + 1 < G ? estart[g + 1] : nnz;
                v0 = vstart[g];
                nv = vstart[g + 1] - v0;
            }
            y[j] = (x[j] >= 0 && x[j] < nv) ? x[j] + (int)v0 : -1;
        }
        if (VEC && e4 + 4 <= e_stop) {
            *reinterpret_cast<int4 *>(ind_g + e4) = make_int4(y[0], y[1], y[2], y[3]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (e4 + j < e_stop) ind_g[e4 + j] = y[j];
        }
    }
}

// graph_T[g] = (sum of t over graph g's vertices) / 3
__global__ void graph_triangles_kernel(const unsigned long long *__restrict__ tacc,
                                       const long long *__restrict__ vstart,
                                       long long *__restrict__ graph_T)
{
    const long long g = blockIdx.x;
    unsigned long long s = 0;
    for (long long v = vstart[g] + threadIdx.x; v < vstart[g + 1]; v += blockDim.x) s += tacc[v];
    auto warp = cg::tiled_partition<32>(cg::this_thread_block());
    s = cg::reduce(warp, s, cg::plus<unsigned long long>());
    __shared__ unsigned long long ws[32];
    if (warp.thread_rank() == 0) ws[warp.meta_group_rank()] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) t += ws[i];
        graph_T[g] = (long long)(t / 3);
    }
}

struct PackRef {
    const long long *off;     // graph-local offsets, off[0] = 0
    const int *ind;           // graph-local ids
};

// Copy separate graphs into one concatenated CSR: off_out[vbase[g] + v] =
// ebase[g] + off_g[v], ind_out[ebase[g] + e] = ind_g[e].  vbase / ebase are
// exclusive prefixes of the graphs' vertex and entry counts (G+1 entries).
__global__ void pack_vertices_kernel(const PackRef *__restrict__ refs,
                                     const long long *__restrict__ vbase,
                                     const long long *__restrict__ ebase, long long G,
                                     long long *__restrict__ off_out, long long total_n,
                                     long long total_nnz)
{
    __shared__ long long s_g0;
    const long long v_begin = (long long)blockIdx.x * kChunk;
    if (threadIdx.x == 0) s_g0 = owner(vbase, G, v_begin);
    __syncthreads();
    long long g = s_g0;
    for (long long v = v_begin + threadIdx.x; v < v_begin + kChunk && v < total_n; v += blockDim.x) {
        while (g + 1 < G && vbase[g + 1] <= v) ++g;
        off_out[v] = ebase[g] + refs[g].off[v - vbase[g]];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) off_out[total_n] = total_nnz;
}

__global__ void pack_entries_kernel(const PackRef *__restrict__ refs,
                                    const long long *__restrict__ ebase, long long G,
                                    int *__restrict__ ind_out, long long total_nnz)
{
    __shared__ long long s_g0;
    const long long e_begin = (long long)blockIdx.x * kChunk;
    if (threadIdx.x == 0) s_g0 = owner(ebase, G, e_begin);
    __syncthreads();
    long long g = s_g0;
    for (long long e = e_begin + threadIdx.x; e < e_begin + kChunk && e < total_nnz; e += blockDim.x) {
        while (g + 1 < G && ebase[g + 1] <= e) ++g;
        ind_out[e] = refs[g].ind[e - ebase[g]];
    }
}

struct BatchPlan {
    Plan inner;               // the union graph's pipeline workspace
    size_t o_estart = 0, o_indg = 0, o_inner = 0, o_ghist = 0, o_scan = 0, o_rend = 0,
           bytes = 0;
};

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// The union graph's pipeline workspace comes first, so that the batch
// workspace starts with its status word (gtc_count_status reads offset 0).
BatchPlan make_batch_plan(long long G, long long total_n, long long total_nnz)
{
    BatchPlan b;
    b.inner = make_plan(total_n, total_nnz, 64, true);
    size_t o = 0;
    b.o_inner = o;  o = align256(o + b.inner.bytes);
    b.o_estart = o; o = align256(o + sizeof(long long) * (size_t)(G + 1));
    b.o_indg = o;   o = align256(o + sizeof(int) * (size_t)(total_nnz + 1));
    // graph-major degree ranks: per-graph bucket histogram and its scan
    b.o_ghist = o;  o = align256(o + sizeof(long long) * (size_t)(G * kSegBuckets + 1));
    b.o_scan = o;   o = align256(o + scan_tmp_bytes(G * kSegBuckets));
    b.o_rend = o;   o = align256(o + sizeof(int) * (size_t)(total_n + 1));
    b.bytes = o;
    return b;
}

}  // namespace
}  // namespace gtc

using namespace gtc;

extern "C" {

gtc_status gtc_batch_workspace_size(int64_t num_graphs, int64_t total_n, int64_t total_nnz,
                                    size_t *bytes)
{
    if (!bytes || num_graphs < 0 || total_n < 0 || total_nnz < 0) return GTC_ERR_INVALID_ARGUMENT;
    if (total_n > 0x7fffffffll) return GTC_ERR_UNSUPPORTED;      // union ids are int32
    *bytes = make_batch_plan(num_graphs, total_n, total_nnz).bytes;
    return GTC_OK;
}

gtc_status gtc_count_batch(int64_t num_graphs, const int64_t *d_vstart, const int64_t *d_off,
                           const int32_t *d_ind, int64_t total_n, int64_t total_nnz,
                           int64_t *d_r, int64_t *d_t, double *d_lcc, int64_t *d_graph_T,
                           void *d_workspace, size_t ws_bytes, const gtc_tuning *tuning,
                           gtc_stream_t stream)
{
    size_t need = 0;
    gtc_status st = gtc_batch_workspace_size(num_graphs, total_n, total_nnz, &need);
    if (st != GTC_OK) return st;
    if (num_graphs == 0) return GTC_OK;
    if (!d_vstart || !d_off || (total_nnz > 0 && !d_ind) || !d_workspace)
        return GTC_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_workspace) & 255) return GTC_ERR_INVALID_ARGUMENT;
    if (ws_bytes < need) return GTC_ERR_WORKSPACE_TOO_SMALL;
    const BatchPlan b = make_batch_plan(num_graphs, total_n, total_nnz);
    char *base = static_cast<char *>(d_workspace);
    long long *estart = reinterpret_cast<long long *>(base + b.o_estart);
    int *ind_g = reinterpret_cast<int *>(base + b.o_indg);
    void *inner = base + b.o_inner;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const long long *vstart = reinterpret_cast<const long long *>(d_vstart);
    const long long *off = reinterpret_cast<const long long *>(d_off);

    RowConfig cfg = pick_row_config(total_n, total_nnz);
    // a batch mixes degree profiles: the warp-per-item kernel unless asked
    // (per-row merges were 24% slower on the 4,096-graph mix)
    cfg.merge_rows = false;
    st = apply_tuning(cfg, tuning);
    if (st != GTC_OK) return st;

    graph_entry_starts<<<(unsigned)div_up<long long>(num_graphs + 1, 256), 256, 0, s>>>(
        off, vstart, num_graphs, estart);
    if (total_nnz > 0)
    {
        const unsigned gb = (unsigned)div_up<long long>(total_nnz, kChunk);
        if ((reinterpret_cast<uintptr_t>(d_ind) & 15) == 0 &&
            (reinterpret_cast<uintptr_t>(ind_g) & 15) == 0)
            globalize_kernel<true><<<gb, 256, 0, s>>>(estart, vstart, num_graphs, d_ind, ind_g,
                                                      total_nnz);
        else
            globalize_kernel<false><<<gb, 256, 0, s>>>(estart, vstart, num_graphs, d_ind, ind_g,
                                                       total_nnz);
    }
    if (cudaGetLastError() != cudaSuccess) return GTC_ERR_CUDA;
    SegRanks seg;
    seg.vstart = vstart;
    seg.num_graphs = num_graphs;
    seg.ghist = reinterpret_cast<long long *>(base + b.o_ghist);
    seg.scan_tmp = base + b.o_scan;
    seg.rank_end = reinterpret_cast<int *>(base + b.o_rend);
    st = run_count<long long>(off, ind_g, total_n, total_nnz, true,
                              reinterpret_cast<long long *>(d_r),
                              reinterpret_cast<long long *>(d_t), d_lcc, nullptr, inner,
                              b.inner.bytes, s, cfg, nullptr, &seg);
    if (st != GTC_OK) return st;
    if (d_graph_T) {
        const unsigned long long *tacc =
            reinterpret_cast<const unsigned long long *>(static_cast<char *>(inner) + b.inner.o_tacc);
        graph_triangles_kernel<<<(unsigned)num_graphs, 256, 0, s>>>(
            tacc, vstart, reinterpret_cast<long long *>(d_graph_T));
    }
    return cudaGetLastError() == cudaSuccess ? GTC_OK : GTC_ERR_CUDA;
}

size_t gtc_batch_pack_scratch_bytes(int64_t num_graphs)
{
    return align256(sizeof(PackRef) * (size_t)(num_graphs > 0 ? num_graphs : 1)) +
           2 * align256(sizeof(long long) * (size_t)(num_graphs + 1));
}

gtc_status gtc_batch_pack(int64_t num_graphs, const void *const *h_off, const void *const *h_ind,
                          const int64_t *h_n, const int64_t *h_nnz, int64_t *d_vstart,
                          int64_t *d_off, int32_t *d_ind, void *d_scratch, size_t scratch_bytes,
                          void *h_staging, gtc_stream_t stream)
{
    if (num_graphs < 0 || (num_graphs > 0 && (!h_off || !h_ind || !h_n || !h_nnz || !d_vstart ||
                                              !d_off || !d_scratch || !h_staging)))
        return GTC_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < gtc_batch_pack_scratch_bytes(num_graphs)) return GTC_ERR_WORKSPACE_TOO_SMALL;
    if (num_graphs == 0) return GTC_OK;
    // host side: descriptor table and prefixes, staged in the caller's pinned
    // buffer (the same layout as the device scratch)
    char *hs = static_cast<char *>(h_staging);
    PackRef *refs = reinterpret_cast<PackRef *>(hs);
    const size_t o_vb = align256(sizeof(PackRef) * (size_t)num_graphs);
    const size_t o_eb = o_vb + align256(sizeof(long long) * (size_t)(num_graphs + 1));
    long long *vb = reinterpret_cast<long long *>(hs + o_vb);
    long long *eb = reinterpret_cast<long long *>(hs + o_eb);
    vb[0] = eb[0] = 0;
    for (int64_t g = 0; g < num_graphs; ++g) {
        if (h_n[g] < 0 || h_nnz[g] < 0 || !h_off[g] || (h_nnz[g] > 0 && !h_ind[g]))
            return GTC_ERR_INVALID_ARGUMENT;
        refs[g].off = static_cast<const long long *>(h_off[g]);
        refs[g].ind = static_cast<const int *>(h_ind[g]);
        vb[g + 1] = vb[g] + h_n[g];
        eb[g + 1] = eb[g] + h_nnz[g];
    }
    const long long total_n = vb[num_graphs], total_nnz = eb[num_graphs];
    if (total_n > 0x7fffffffll) return GTC_ERR_UNSUPPORTED;
    if (total_nnz > 0 && !d_ind) return GTC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t table_bytes = o_eb + sizeof(long long) * (size_t)(num_graphs + 1);
    if (cudaMemcpyAsync(d_scratch, h_staging, table_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return GTC_ERR_CUDA;
    char *ds = static_cast<char *>(d_scratch);
    const PackRef *d_refs = reinterpret_cast<const PackRef *>(ds);
    const long long *d_vb = reinterpret_cast<const long long *>(ds + o_vb);
    const long long *d_eb = reinterpret_cast<const long long *>(ds + o_eb);
    if (cudaMemcpyAsync(d_vstart, d_vb, sizeof(long long) * (size_t)(num_graphs + 1),
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return GTC_ERR_CUDA;
    pack_vertices_kernel<<<(unsigned)div_up<long long>(total_n + 1, kChunk), 256, 0, s>>>(
        d_refs, d_vb, d_eb, num_graphs, reinterpret_cast<long long *>(d_off), total_n, total_nnz);
    if (total_nnz > 0)
        pack_entries_kernel<<<(unsigned)div_up<long long>(total_nnz, kChunk), 256, 0, s>>>(
            d_refs, d_eb, num_graphs, d_ind, total_nnz);
    return cudaGetLastError() == cudaSuccess ? GTC_OK : GTC_ERR_CUDA;
}

}  // extern "C"
