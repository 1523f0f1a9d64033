// ref_gpu_shim.cu -- extern "C" entry point over the reference's own GPU
// kernel (count_all_trianglesGPU via kernelCall), compiled for sm_100a from the
// reference's sources by oracle/Makefile (target `ref`).  TEST INFRASTRUCTURE
// ONLY: a second oracle for the GPU tests.  Only threads-per-intersection 1 is
// exposed: with tpi=1 the Merge Path search never runs (diagonal 0 starts
// "found"), so the kernel reads only inside each adjacency list, and its
// shared-memory hand-off between lanes (src/clusteringCount.cu:192,205-209),
// which races under independent thread scheduling, is never used.
#include <cstdint>
#include <cuda_runtime.h>

// Declaration of the reference host dispatcher, plain overload
// (src/clusteringCount.cu:415-467, instantiated at :518-524).
template <typename T>
void kernelCall(unsigned int numberBlocks, unsigned int numberThreads,
                const T nv, T const *const __restrict__ d_off,
                T const *const __restrict__ d_ind,
                T *const __restrict__ outPutTriangles,
                const T threads_per_block, const T number_blocks,
                const T shifter);

extern "C" int ref_gpu_count_i64(unsigned int blocks, unsigned int block_size,
                                 int64_t nv, const int64_t *d_off,
                                 const int64_t *d_ind, int64_t *d_out)
{
    // tpi = 1: groups per block = block_size, shift = log2(1) = 0
    // (src/gpurun.cu:31-35).
    kernelCall<int64_t>(blocks, block_size, nv, d_off, d_ind, d_out, 1,
                        (int64_t)block_size, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    e = cudaDeviceSynchronize();
    return (int)e;
}
