// A caller written against the reference's kernelCall<T> operator
// (src/gpurun.cu:31-37 of the reference): it must compile and link against
// libgtc_b200.so through include/gtc_b200_kernelcall.hpp unchanged.
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "gtc_b200_kernelcall.hpp"

template <typename T>
void run_like_the_reference(unsigned blocks, unsigned blockSize, T vertexCount,
                            const T *dOffset, const T *dIndex, T *dTriangle,
                            T threadPerInt)
{
    T intsctnPerBlock = blockSize / threadPerInt;
    T threadShift = (T)std::log2((double)threadPerInt);
    kernelCall(blocks, blockSize, vertexCount, dOffset, dIndex, dTriangle, threadPerInt,
               intsctnPerBlock, threadShift);
}

int main(int argc, char **)
{
    if (argc > 1) {   // never run without a device; the test only links
        run_like_the_reference<int64_t>(1024, 256, 0, nullptr, nullptr, nullptr, 1);
        run_like_the_reference<int32_t>(1024, 256, 0, nullptr, nullptr, nullptr, 1);
        std::printf("%s\n", gtc_status_string(gtc_kernelCall_status()));
    }
    return 0;
}
