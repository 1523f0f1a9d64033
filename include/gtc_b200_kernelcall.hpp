// gtc_b200_kernelcall.hpp -- header-only C++ drop-in for the reference's
// host operator kernelCall<T> (declared in include/clusteringCount.cuh:92-104
// and defined in src/clusteringCount.cu:361-467 of ogreen/GpuTriangleCounting).
//
// Same template name, argument list and meaning, instantiated for int32_t and
// int64_t like the reference (src/clusteringCount.cu:510-542).  A caller such
// as the reference's singleParamTestGPURun (src/gpurun.cu:31-37) compiles
// unchanged after including this header instead of clusteringCount.cuh and
// linking libgtc_b200.so:
//
//   kernelCall(blocks, blockSize, vertexCount, dOffset, dIndex, dTriangle,
//              threadsPerIntsctn, intsctnPerBlock, threadShift);
//   cudaDeviceSynchronize();
//
// out[v] = sum over u in N(v) of |N(v) ∩ N(u)| (= 2 x triangles at v).  The
// tuning arguments are hints.  An unsupported block size launches nothing, as
// in the reference; gtc_kernelCall_status() (or gtc_compat_last_status())
// reports that and every other failure.
#pragma once

#include <cstdint>

#include "gtc_b200.h"

template <typename T>
void kernelCall(unsigned int numberBlocks, unsigned int numberThreads, const T nv,
                T const *const d_off, T const *const d_ind, T *const outPutTriangles,
                const T threads_per_block, const T number_blocks, const T shifter);

template <typename T>
void kernelCall(unsigned int numberBlocks, unsigned int numberThreads, const T nv,
                T const *const vertex, T const *const d_off, T const *const d_ind,
                T *const outPutTriangles, const T threads_per_block,
                const T number_blocks, const T shifter);

template <>
inline void kernelCall<int64_t>(unsigned int numberBlocks, unsigned int numberThreads,
                                const int64_t nv, int64_t const *const d_off,
                                int64_t const *const d_ind, int64_t *const out,
                                const int64_t tpi, const int64_t groups,
                                const int64_t shifter)
{
    gtc_kernelCall_i64(numberBlocks, numberThreads, nv, d_off, d_ind, out, tpi, groups, shifter);
}

template <>
inline void kernelCall<int32_t>(unsigned int numberBlocks, unsigned int numberThreads,
                                const int32_t nv, int32_t const *const d_off,
                                int32_t const *const d_ind, int32_t *const out,
                                const int32_t tpi, const int32_t groups,
                                const int32_t shifter)
{
    gtc_kernelCall_i32(numberBlocks, numberThreads, nv, d_off, d_ind, out, tpi, groups, shifter);
}

template <>
inline void kernelCall<int64_t>(unsigned int numberBlocks, unsigned int numberThreads,
                                const int64_t nv, int64_t const *const vertex,
                                int64_t const *const d_off, int64_t const *const d_ind,
                                int64_t *const out, const int64_t tpi, const int64_t groups,
                                const int64_t shifter)
{
    gtc_kernelCall_vertex_i64(numberBlocks, numberThreads, nv, vertex, d_off, d_ind, out, tpi,
                              groups, shifter);
}

template <>
inline void kernelCall<int32_t>(unsigned int numberBlocks, unsigned int numberThreads,
                                const int32_t nv, int32_t const *const vertex,
                                int32_t const *const d_off, int32_t const *const d_ind,
                                int32_t *const out, const int32_t tpi, const int32_t groups,
                                const int32_t shifter)
{
    gtc_kernelCall_vertex_i32(numberBlocks, numberThreads, nv, vertex, d_off, d_ind, out, tpi,
                              groups, shifter);
}

inline gtc_status gtc_kernelCall_status() { return gtc_compat_last_status(); }
