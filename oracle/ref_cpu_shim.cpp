// ref_cpu_shim.cpp -- extern "C" entry points over the reference's own CPU
// triangle count, compiled unchanged from the reference's sources by
// oracle/Makefile (target `ref`).  TEST INFRASTRUCTURE ONLY: the test-suite and
// the CPU-baseline / reference arm of bench.py call it as the checker and the
// timed reference; the product library never links it.
#include <chrono>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif

// Declarations of the reference templates (src/clusteringCount.cpp:50-70 and
// :125-155; explicit instantiations at :260-294 of the same file).
template <typename T>
void count_all_trianglesCPU(const T nv, const T *off, const T *ind,
                            int64_t *triNE, int64_t *allTriangles);
template <typename T>
void count_all_trianglesCPU(const T nv, const T *vertexList, const T *off,
                            const T *ind, int64_t *triNE,
                            int64_t *allTriangles);

extern "C" {

// Serial whole-graph call: per-edge triNE (CSR order) and its total.
int64_t ref_cpu_tri_ne_i64(int64_t nv, const int64_t *off, const int64_t *ind,
                           int64_t *triNE)
{
    int64_t all = 0;
    count_all_trianglesCPU<int64_t>(nv, off, ind, triNE, &all);
    return all;
}

int64_t ref_cpu_tri_ne_i32(int32_t nv, const int32_t *off, const int32_t *ind,
                           int64_t *triNE)
{
    int64_t all = 0;
    count_all_trianglesCPU<int32_t>(nv, off, ind, triNE, &all);
    return all;
}

// All-core form: the vertex-list overload called one vertex at a time under
// OpenMP (dynamic, 64).  Each call writes that vertex's triNE slice in place,
// so the arithmetic is the reference's own.  r[v] receives the row sum of
// triNE (what the reference GPU kernel stores in out[v]).  `vertices` is the
// list of rows to process (NULL = all rows 0..nv-1, count = nv); returns the
// sum of triNE over the processed rows.
int64_t ref_cpu_rows_omp_i64(int64_t nv, const int64_t *off,
                             const int64_t *ind, const int64_t *vertices,
                             int64_t count, int64_t *triNE, int64_t *r,
                             int threads)
{
    int64_t total = 0;
    if (!vertices) count = nv;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total) num_threads(threads)
#endif
    for (int64_t q = 0; q < count; ++q) {
        int64_t v = vertices ? vertices[q] : q;
        int64_t row_sum = 0;
        count_all_trianglesCPU<int64_t>(1, &v, off, ind, triNE + off[v],
                                        &row_sum);
        if (r) r[v] = row_sum;
        total += row_sum;
    }
    (void)threads;
    return total;
}

// Timed all-core form on an int32 CSR (the workloads' layout; the reference
// instantiates count_all_trianglesCPU<int32_t>, src/clusteringCount.cpp:260-294).
// The rows are grouped into units -- unit u holds the rows
// unit_rows[unit_off[u] .. unit_off[u+1]) -- and the listed units run under
// OpenMP (dynamic, 1), each by one thread, row by row through the
// vertex-list overload.  unit_ns[k] receives the elapsed nanoseconds of unit
// units[k]; r[v] the row sum of triNE for every row run.  Returns the sum of
// triNE over the rows run.
int64_t ref_cpu_units_timed_i32(int32_t nv, const int32_t *off, const int32_t *ind,
                                const int64_t *unit_rows, const int64_t *unit_off,
                                const int64_t *units, int64_t n_units, int64_t *triNE,
                                int64_t *r, int64_t *unit_ns, int threads)
{
    int64_t total = 0;
    (void)nv;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(threads)
#endif
    for (int64_t k = 0; k < n_units; ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        const int64_t u = units[k];
        for (int64_t q = unit_off[u]; q < unit_off[u + 1]; ++q) {
            int32_t v = (int32_t)unit_rows[q];
            int64_t row_sum = 0;
            count_all_trianglesCPU<int32_t>(1, &v, off, ind, triNE + off[v], &row_sum);
            if (r) r[v] = row_sum;
            total += row_sum;
        }
        unit_ns[k] = std::chrono::duration_cast<std::chrono::nanoseconds>(
                         std::chrono::steady_clock::now() - t0).count();
    }
    (void)threads;
    return total;
}

int ref_cpu_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
