/*
 * gtc_b200.h -- C ABI of the B200 per-vertex triangle counter.
 *
 * Drop-in boundary for the reference's GPU operator (ogreen/GpuTriangleCounting):
 * a symmetric CSR goes in, per-vertex triangle counts, local clustering
 * coefficients and the global count come out.  Every entry point returns a
 * gtc_status (never exits), works on caller-owned device memory, and takes an
 * explicit CUDA stream (a cudaStream_t passed as void*; NULL = legacy default
 * stream).  The library is built for sm_100a only.
 *
 * Input contract (checked by gtc_validate_csr, not by the counting calls):
 *   off[n+1] non-decreasing, off[0] = 0, off[n] = nnz   (int32 or int64)
 *   ind[nnz] int32 in [0, n), each row strictly ascending, no self-loops,
 *   symmetric (v in N(u) <=> u in N(v)).
 *
 * Output semantics (reference: src/clusteringCount.cu:314-359 and
 * src/clusteringCount.cpp:50-70):
 *   r[v]   = sum over u in N(v) of |N(v) ∩ N(u)|  = 2 t(v)   (what the
 *            reference kernel stores in out[v])
 *   t[v]   = number of triangles through v
 *   lcc[v] = (double)r[v] / (double)(d(v)(d(v)-1)),  0.0 when d(v) < 2
 *   global[0] = T (triangles), global[1] = 3T (the dest<src oriented sum of
 *   README.md:6-10), global[2] = 6T (sum of r, "totalTriangleCount" printed by
 *   src/gpurun.cu:40-49).
 */
#ifndef GTC_B200_H
#define GTC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gtc_status {
    GTC_OK = 0,
    GTC_ERR_INVALID_ARGUMENT = 1,   /* null pointer, negative size, bad enum   */
    GTC_ERR_INVALID_CSR = 2,        /* input violates the CSR contract         */
    GTC_ERR_WORKSPACE_TOO_SMALL = 3,
    GTC_ERR_CUDA = 4,               /* a CUDA runtime call failed              */
    GTC_ERR_OUT_OF_MEMORY = 5,
    GTC_ERR_UNSUPPORTED = 6,        /* e.g. no sm_100 device                   */
    GTC_ERR_TIMEOUT = 7,            /* a bounded device wait ran out           */
    GTC_ERR_CAPACITY = 8,           /* a fixed-capacity limit was exceeded     */
    GTC_ERR_BUSY = 9                /* resource in use / admission refused     */
} gtc_status;

typedef enum gtc_mode {
    /* per-vertex counts (r, t, lcc) plus the global count */
    GTC_MODE_PLAIN = 0,
    /* global count only: the reference README's dest<src mode, no
       per-vertex bookkeeping (README.md:6-10) */
    GTC_MODE_ORIENTED = 1
} gtc_mode;

/* Reasons reported by gtc_validate_csr (0 = valid). */
typedef enum gtc_csr_reason {
    GTC_CSR_OK = 0,
    GTC_CSR_BAD_OFFSETS = 1,        /* off[0] != 0, off[n] != nnz or decreasing */
    GTC_CSR_INDEX_RANGE = 2,
    GTC_CSR_SELF_LOOP = 3,
    GTC_CSR_UNSORTED_OR_DUPLICATE = 4,
    GTC_CSR_ASYMMETRIC = 5
} gtc_csr_reason;

typedef void *gtc_stream_t;  /* a cudaStream_t */

const char *gtc_status_string(gtc_status s);

/* Library / device information: writes the sm count, and the compute
   capability major*10+minor of the current device. */
gtc_status gtc_device_info(int *sm_count, int *cc);

/* Bytes of device workspace gtc_count needs for a graph of this size.
   off_bits is 32 or 64 (the width of the offsets array). */
gtc_status gtc_workspace_size(int64_t n, int64_t nnz, int off_bits,
                              gtc_mode mode, size_t *bytes);

/*
 * Count triangles.  Replaces kernelCall<T> + thrust::reduce
 * (src/clusteringCount.cu:415-467, src/gpurun.cu:36-41).
 *   d_off       device, n+1 offsets, int32 (off_bits 32) or int64 (64)
 *   d_ind       device, nnz int32 neighbour ids
 *   d_r, d_t    device int64[n] or NULL (PLAIN mode only)
 *   d_lcc       device double[n] or NULL (PLAIN mode only)
 *   d_global    device int64[3] or NULL: {T, 3T, 6T}
 *   d_workspace device, >= gtc_workspace_size bytes, 256-byte aligned
 * Asynchronous on `stream`; the caller synchronises.  The counting calls do
 * not validate the input (like the reference's kernel), but a neighbour id
 * outside [0, n) is never dereferenced: it is skipped and recorded in the
 * workspace, and gtc_count_status then reports GTC_ERR_INVALID_CSR (the
 * counts of such a graph are meaningless).
 */
gtc_status gtc_count(const void *d_off, int off_bits, const int32_t *d_ind,
                     int64_t n, int64_t nnz, gtc_mode mode,
                     int64_t *d_r, int64_t *d_t, double *d_lcc,
                     int64_t *d_global, void *d_workspace, size_t ws_bytes,
                     gtc_stream_t stream);

/*
 * Device-side error report of the last count that used this workspace
 * (gtc_count, gtc_count_tuned or gtc_count_batch; the status word is the
 * workspace's first 4 bytes and each count clears it when it starts).
 * Synchronous: waits for `stream`, then returns GTC_OK, or
 * GTC_ERR_INVALID_CSR if a neighbour id outside its graph's vertex range was
 * met.  h_bits (nullable) receives the raw error bits.  The reference has no
 * counterpart: its launches are unchecked (include/clusteringCount.cuh:4-11,
 * src/clusteringCount.cu:410-412).
 */
gtc_status gtc_count_status(const void *d_workspace, size_t ws_bytes,
                            gtc_stream_t stream, uint32_t *h_bits);

/*
 * Launch-shape overrides for gtc_count_tuned (0 in any field = the library's
 * choice).  Used by the autotuner, which replaces the reference's
 * block-size x threads-per-intersection sweep (src/gpurun.cu:115-176,
 * src/param.cu:2-6).  None of them changes the result.
 *   group        lanes that share one apex row in the group kernel: 4, 8,
 *                16 or 32; rows whose forward list is longer than
 *                4*group go to the block kernel
 *   item_len     adjacency entries per warp work item (a power of two, 32 .. 32768)
 *   big_chunk    adjacency entries per block-kernel work item (32 .. 32768)
 *   big_hash_max longest forward list the block kernel hashes in shared
 *                memory (<= 2048); longer lists are binary-searched in place
 *   labels       how forward lists name vertices: 1 = vertex ids (order by
 *                (degree, id)), 2 = degree ranks (vertices counting-sorted
 *                by degree, lists sorted by rank, block kernel on a rank
 *                bitmap); the library picks ranks for mean degree > 24
 *   region       warp-kernel hash slots per forward-list member: 2 or 4 (the
 *                library picks 2 for mean degree <= 24, else 4)
 *   rows         the group kernel's form: 1 = warp per work item with per-row
 *                hash regions, 2 = per-row merges of id-ordered forward lists
 *                (vertex-id labels only; with labels = 2 it is rejected, with
 *                labels = 0 it implies vertex ids).  The library picks 2 for
 *                single graphs with vertex-id labels and at least 2^18
 *                vertices, else 1
 */
typedef struct gtc_tuning {
    int group;
    int item_len;
    int big_chunk;
    int big_hash_max;
    int labels;
    int region;
    int rows;
} gtc_tuning;

/* Values of gtc_tuning.labels. */
enum { GTC_LABELS_AUTO = 0, GTC_LABELS_VERTEX_ID = 1, GTC_LABELS_DEGREE_RANK = 2 };
/* Values of gtc_tuning.rows. */
enum { GTC_ROWS_AUTO = 0, GTC_ROWS_HASH = 1, GTC_ROWS_MERGE = 2 };

/*
 * What gtc_count_tuned would run for this graph size and tuning (NULL = the
 * library's choice), without touching the device: *launches = kernels of one
 * count (with every output requested), *labels = GTC_LABELS_VERTEX_ID or
 * GTC_LABELS_DEGREE_RANK.  No counterpart in the reference (introspection).
 */
gtc_status gtc_count_launches(int64_t n, int64_t nnz, gtc_mode mode,
                              const gtc_tuning *tuning, int *launches, int *labels);

gtc_status gtc_count_tuned(const void *d_off, int off_bits,
                           const int32_t *d_ind, int64_t n, int64_t nnz,
                           gtc_mode mode, int64_t *d_r, int64_t *d_t,
                           double *d_lcc, int64_t *d_global,
                           void *d_workspace, size_t ws_bytes,
                           gtc_stream_t stream, const gtc_tuning *tuning);

/*
 * Diagnostic: one synchronous per-vertex count on the legacy default stream
 * with CUDA events between the pipeline phases; writes the device time in ms
 * of {forward-list build, group kernel, block kernel, epilogue} to h_ms[4].
 * tuning: as for gtc_count_tuned (NULL = the library's choice).  Stands in for
 * the reference's chrono timing around launch + sync (src/gpurun.cu:17-47,
 * timedKernelCall :469-508).
 */
gtc_status gtc_count_phase_times(const void *d_off, int off_bits,
                                 const int32_t *d_ind, int64_t n, int64_t nnz,
                                 void *d_workspace, size_t ws_bytes,
                                 float *h_ms, const gtc_tuning *tuning);

/*
 * gtc_count with no device allocation at all, for callers that cannot
 * allocate when they count (a serving loop that reserved its memory at start-up,
 * a plug-in whose host framework owns the device memory, or a caller that must
 * avoid the synchronisation cudaMalloc/cudaFree can cause).  This entry point
 * has no counterpart in the reference.  The pipeline's scratch lives in a
 * fixed 32 MiB array inside the library: graphs whose gtc_workspace_size
 * exceeds it are rejected with GTC_ERR_CAPACITY.  Every device that loads the
 * library holds the array until exit.  All calls on a device share it, so
 * calls that overlap on the GPU race and must be serialised.  The first call
 * on each device looks up the array's address; make it before any stream
 * capture.  The looked-up address is kept for the life of the process: after
 * a cudaDeviceReset on that device it is stale, so a process that resets a
 * device must not call this entry point on it again.  Arguments and outputs
 * as gtc_count; asynchronous on `stream`.
 */
gtc_status gtc_count_noalloc(const void *d_off, int off_bits,
                             const int32_t *d_ind, int64_t n, int64_t nnz,
                             gtc_mode mode, int64_t *d_r, int64_t *d_t,
                             double *d_lcc, int64_t *d_global,
                             gtc_stream_t stream);

/*
 * Per-vertex counts for a vertex subset: d_out[k] = r(d_vertex[k]) for
 * k < count.  Replaces the vertex-list kernelCall overload
 * (src/clusteringCount.cu:361-413, kernel :266-312).  Like the reference it
 * reads only the listed rows and their neighbours' rows, so it needs neither
 * the graph size nor a workspace.  Asynchronous on `stream`.
 */
gtc_status gtc_count_subset(const void *d_off, int off_bits,
                            const int32_t *d_ind, const int32_t *d_vertex,
                            int64_t count, int64_t *d_out,
                            gtc_stream_t stream);

/*
 * Batched counting: many independent graphs in one pipeline run (no
 * counterpart in the reference, whose host path counts one graph per
 * kernelCall, src/gpurun.cu:2-56).
 *   d_vstart[G+1]   int64 vertex starts of the graphs in the concatenated
 *                   vertex space (d_vstart[0] = 0, d_vstart[G] = total_n)
 *   d_off[total_n+1] int64 offsets into the concatenated adjacency
 *   d_ind[total_nnz] int32 graph-local neighbour ids (0 .. n_g-1)
 *   d_r, d_t, d_lcc  per-vertex outputs over the concatenated vertex space
 *                   (nullable); d_graph_T[G] triangles per graph (nullable)
 * Every graph obeys the single-graph contract; total_n < 2^31.  The result
 * for each graph is exactly the one gtc_count gives for it alone.
 * Asynchronous on `stream`; capturable in a CUDA graph after one warm-up call.
 */
gtc_status gtc_batch_workspace_size(int64_t num_graphs, int64_t total_n,
                                    int64_t total_nnz, size_t *bytes);
gtc_status gtc_count_batch(int64_t num_graphs, const int64_t *d_vstart,
                           const int64_t *d_off, const int32_t *d_ind,
                           int64_t total_n, int64_t total_nnz, int64_t *d_r,
                           int64_t *d_t, double *d_lcc, int64_t *d_graph_T,
                           void *d_workspace, size_t ws_bytes,
                           const gtc_tuning *tuning, gtc_stream_t stream);

/*
 * Gather separate device-resident graphs (graph-local int64 offsets and int32
 * ids; host arrays of their device pointers and sizes) into the batched
 * layout above.  d_scratch needs gtc_batch_pack_scratch_bytes(G) bytes;
 * h_staging is pinned host memory of the same size that must stay untouched
 * until the stream has passed this call.
 */
size_t gtc_batch_pack_scratch_bytes(int64_t num_graphs);
gtc_status gtc_batch_pack(int64_t num_graphs, const void *const *h_off,
                          const void *const *h_ind, const int64_t *h_n,
                          const int64_t *h_nnz, int64_t *d_vstart,
                          int64_t *d_off, int32_t *d_ind, void *d_scratch,
                          size_t scratch_bytes, void *h_staging,
                          gtc_stream_t stream);

/*
 * Check the CSR input contract on the device.  Synchronous: writes a
 * gtc_csr_reason to *h_reason and returns GTC_OK (the status reports only
 * call failures; an invalid graph is reported through *h_reason).
 * Workspace: gtc_validate_workspace_size(n, nnz) bytes, 256-byte aligned.
 */
size_t gtc_validate_workspace_size(int64_t n, int64_t nnz);
gtc_status gtc_validate_csr(const void *d_off, int off_bits,
                            const int32_t *d_ind, int64_t n, int64_t nnz,
                            void *d_workspace, size_t ws_bytes,
                            int32_t *h_reason, gtc_stream_t stream);

/*
 * Reference-compatible operator (src/clusteringCount.cu:415-467): the plain
 * kernelCall<T> overload with the same argument list and meaning.
 * numberBlocks, threads_per_block (tpi), number_blocks (groups per block)
 * and shifter are accepted as tuning hints and ignored.  As in the
 * reference, an unsupported numberThreads (not one of 32, 64, 96, 128, 192,
 * 256, 512, 1024) launches nothing; unlike the reference, that and every
 * other failure is recorded and can be read with gtc_compat_last_status().
 * out[v] = r(v) in type T; asynchronous on the legacy default stream, the
 * caller synchronises (src/gpurun.cu:38).  Device workspace is allocated
 * internally on first use and cached per device.
 */
void gtc_kernelCall_i64(unsigned int numberBlocks, unsigned int numberThreads,
                        int64_t nv, const int64_t *d_off,
                        const int64_t *d_ind, int64_t *outPutTriangles,
                        int64_t threads_per_block, int64_t number_blocks,
                        int64_t shifter);
void gtc_kernelCall_i32(unsigned int numberBlocks, unsigned int numberThreads,
                        int32_t nv, const int32_t *d_off,
                        const int32_t *d_ind, int32_t *outPutTriangles,
                        int32_t threads_per_block, int32_t number_blocks,
                        int32_t shifter);
/* Vertex-list overload (src/clusteringCount.cu:361-413): out[k] =
   r(vertex[k]) for k < nv, where nv counts the listed vertices (as in the
   reference).  Same hint and error behaviour as the plain overload. */
void gtc_kernelCall_vertex_i64(unsigned int numberBlocks,
                               unsigned int numberThreads, int64_t nv,
                               const int64_t *vertex, const int64_t *d_off,
                               const int64_t *d_ind, int64_t *outPutTriangles,
                               int64_t threads_per_block,
                               int64_t number_blocks, int64_t shifter);
void gtc_kernelCall_vertex_i32(unsigned int numberBlocks,
                               unsigned int numberThreads, int32_t nv,
                               const int32_t *vertex, const int32_t *d_off,
                               const int32_t *d_ind, int32_t *outPutTriangles,
                               int32_t threads_per_block,
                               int32_t number_blocks, int32_t shifter);
/* Status of this host thread's last kernelCall shim call: the host-side
   outcome, and -- when that call launched a count -- the device error word of
   that count, read after a copy on the legacy default stream (so this call
   waits for the count; GTC_ERR_INVALID_CSR when a neighbour id was outside
   [0, nv)).  Like the reference, the shims are not re-entrant across host
   threads on one device: they share one cached workspace. */
gtc_status gtc_compat_last_status(void);
/* Releases the compat layer's cached workspace on the current device. */
gtc_status gtc_compat_release(void);

#ifdef __cplusplus
}
#endif
#endif /* GTC_B200_H */
