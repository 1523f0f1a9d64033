/*
 * tc_oracle.c -- CPU restatement of the reference's per-vertex triangle count.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only the test-suite, the smoke check and the CPU-baseline leg
 * of bench.py use it, and only as the checker.
 *
 * Parity is pinned two ways: (1) every function here is checked against the
 * reference's own count_all_trianglesCPU compiled from its sources
 * (oracle/Makefile target `ref`, output in oracle/_ref/), and (2) against the
 * closed-form and reference-generated fixtures in tests/golden/.
 *
 * Layout: int64 CSR offsets (n+1), int32 adjacency (nnz).  Outputs are int64.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/*
 * Size of the intersection of two ascending adjacency lists, skipping the
 * list owner's own id in each list.  Restates count_intersectionsReg
 * (src/clusteringCount.cpp:2-48): early exit on empty or disjoint ranges
 * (:9-10), self-entry skip per list (:19-32), equal step (:34-36) and the
 * linear skip-ahead on the smaller head (:37-45).
 */
static int64_t isect_count(int32_t a_id, int64_t a_len, const int32_t *a,
                           int32_t b_id, int64_t b_len, const int32_t *b)
{
    if (a_len == 0 || b_len == 0) return 0;
    if (a[a_len - 1] < b[0] || b[b_len - 1] < a[0]) return 0;
    int64_t i = 0, j = 0, hits = 0;
    for (;;) {
        if (i >= a_len || j >= b_len) break;
        int32_t x = a[i], y = b[j];
        if (x == a_id) {               /* skip own id in a */
            if (++i >= a_len) break;
            x = a[i];
        }
        if (y == b_id) {               /* skip own id in b */
            if (++j >= b_len) break;
            y = b[j];
        }
        if (x == y) {
            ++i; ++j; ++hits;
        } else if (x < y) {
            ++i;
            while (i < a_len && a[i] < y) ++i;
        } else {
            ++j;
            while (j < b_len && b[j] < x) ++j;
        }
    }
    return hits;
}

/*
 * Per directed edge count, CSR order: tri_ne[e] = |N(src) ∩ N(dst)| for edge
 * e = (src -> ind[e]).  Restates count_all_trianglesCPU
 * (src/clusteringCount.cpp:50-70) including its running total (:66,69).
 * Returns the total (Σ tri_ne = 6T on a simple symmetric graph).
 */
int64_t oracle_tri_ne(int64_t nv, const int64_t *off, const int32_t *ind,
                      int64_t *tri_ne)
{
    int64_t sum = 0;
    for (int64_t s = 0; s < nv; ++s) {
        int64_t s_len = off[s + 1] - off[s];
        for (int64_t e = off[s]; e < off[s + 1]; ++e) {
            int32_t d = ind[e];
            int64_t d_len = off[(int64_t)d + 1] - off[d];
            tri_ne[e] = isect_count((int32_t)s, s_len, ind + off[s],
                                    d, d_len, ind + off[d]);
            sum += tri_ne[e];
        }
    }
    return sum;
}

/*
 * Per-vertex outputs from one pass: r[v] = Σ_{e in row v} tri_ne[e] (the
 * value the reference GPU kernel stores in out[v],
 * src/clusteringCount.cu:333-357), t[v] = r[v]/2, lcc[v] = r / (d (d-1)) in
 * fp64 with d(d-1) formed in int64 (0 for d < 2).  Any output may be NULL.
 * Rows are independent, so with OpenMP the loop is split over vertices
 * (dynamic, 64) exactly like the reference's vertex-list overload
 * (src/clusteringCount.cpp:125-155) called one vertex at a time.
 * Returns Σ r.
 */
int64_t oracle_per_vertex(int64_t nv, const int64_t *off, const int32_t *ind,
                          int64_t *r, int64_t *t, double *lcc, int threads)
{
    int64_t total = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total) num_threads(threads)
#endif
    for (int64_t s = 0; s < nv; ++s) {
        int64_t s_len = off[s + 1] - off[s];
        int64_t acc = 0;
        for (int64_t e = off[s]; e < off[s + 1]; ++e) {
            int32_t d = ind[e];
            int64_t d_len = off[(int64_t)d + 1] - off[d];
            acc += isect_count((int32_t)s, s_len, ind + off[s],
                               d, d_len, ind + off[d]);
        }
        if (r) r[s] = acc;
        if (t) t[s] = acc / 2;
        if (lcc) {
            int64_t pairs = s_len * (s_len - 1);
            lcc[s] = (s_len < 2) ? 0.0 : (double)acc / (double)pairs;
        }
        total += acc;
    }
    (void)threads;
    return total;
}

/*
 * Global count in the dest<src oriented mode (README.md:6-10): the sum of
 * tri_ne over edges whose destination is below the source.  On a simple
 * symmetric graph this is 3T; the README's "multiply by 2" gives Σ r = 6T.
 */
int64_t oracle_oriented_sum(int64_t nv, const int64_t *off, const int32_t *ind,
                            int threads)
{
    int64_t total = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total) num_threads(threads)
#endif
    for (int64_t s = 0; s < nv; ++s) {
        int64_t s_len = off[s + 1] - off[s];
        for (int64_t e = off[s]; e < off[s + 1]; ++e) {
            int32_t d = ind[e];
            if (d >= s) continue;
            int64_t d_len = off[(int64_t)d + 1] - off[d];
            total += isect_count((int32_t)s, s_len, ind + off[s],
                                 d, d_len, ind + off[d]);
        }
    }
    (void)threads;
    return total;
}

/*
 * Per-vertex counts for a vertex subset: out[k] = r(vertex[k]).  Restates the
 * vertex-list overload (src/clusteringCount.cu:266-312 on the GPU,
 * src/clusteringCount.cpp:125-155 on the CPU).
 */
void oracle_subset(int64_t k, const int32_t *vertex, const int64_t *off,
                   const int32_t *ind, int64_t *out, int threads)
{
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
#endif
    for (int64_t q = 0; q < k; ++q) {
        int64_t s = vertex[q];
        int64_t s_len = off[s + 1] - off[s];
        int64_t acc = 0;
        for (int64_t e = off[s]; e < off[s + 1]; ++e) {
            int32_t d = ind[e];
            int64_t d_len = off[(int64_t)d + 1] - off[d];
            acc += isect_count((int32_t)s, s_len, ind + off[s],
                               d, d_len, ind + off[d]);
        }
        out[q] = acc;
    }
    (void)threads;
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
