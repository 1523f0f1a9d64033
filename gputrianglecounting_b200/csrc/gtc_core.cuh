// gtc_core.cuh -- host interface of the single-graph counting pipeline.
#pragma once

#include "gtc_internal.cuh"

namespace gtc {

// Launch shape of the group-per-row kernel (chosen per graph by the host,
// overridable by the autotuner).
struct RowConfig {
    int group = 32;       // lanes per apex row: 4, 8, 16 or 32
    int item_len = 512;   // adjacency entries per dynamic work item
    int big_chunk = 2048; // adjacency entries per block-kernel item
    int big_hash_max = kBigHashMaxFdeg;  // longest list hashed by the block kernel
    bool rank_labels = true;  // label vertices by degree rank (skewed graphs)
    int region_mult = 4;      // warp kernel: table slots per forward member (2 or 4);
                              // low-degree graphs fit twice the rows per batch with 2
    bool merge_rows = false;  // vertex-id labels: lane-per-row merge kernel in place of
                              // the warp-per-item kernel
};

// Kernel launches of one run_count with this configuration (the epilogue
// kernels counted as launched).
int launches_per_count(const RowConfig &cfg, bool per_vertex, long long n);

// Apply caller overrides (gtc_tuning, 0 = keep) to cfg; GTC_ERR_INVALID_ARGUMENT
// for a value outside the documented ranges.
gtc_status apply_tuning(RowConfig &cfg, const gtc_tuning *tuning);

// Optional CUDA events recorded between the pipeline phases:
// ev[0] start, ev[1] forward lists built, ev[2] group kernel done,
// ev[3] block kernel done, ev[4] epilogue done.
struct CountTimings {
    cudaEvent_t ev[5];
};

// Degree-rank labels for a batch: the vertex space is cut into graphs
// (vstart[0..G]) and ranks are made graph-major -- graph g's vertices take the
// ranks vstart[g] .. vstart[g+1]-1 in ascending degree order -- so that an
// apex's forward list spans only its own graph's ranks.  ghist holds
// G * kSegBuckets + 1 int64 counters, scan_tmp scan_tmp_bytes(G * kSegBuckets),
// rank_end n ints (the end of each vertex's graph's ranks).
struct SegRanks {
    const long long *vstart = nullptr;
    long long num_graphs = 0;
    long long *ghist = nullptr;
    void *scan_tmp = nullptr;
    int *rank_end = nullptr;
};

Plan make_plan(long long n, long long nnz, int off_bits, bool per_vertex);
RowConfig pick_row_config(long long n, long long nnz);

template <typename OffT>
gtc_status run_count(const OffT *off, const int *ind, long long n, long long nnz,
                     bool per_vertex, long long *r, long long *t, double *lcc,
                     long long *global, void *ws, size_t ws_bytes,
                     cudaStream_t stream, const RowConfig &cfg,
                     CountTimings *timing, const SegRanks *seg = nullptr);

}  // namespace gtc
