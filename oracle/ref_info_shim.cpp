// ref_info_shim.cpp -- extern "C" entry point over the reference's own `.info`
// reader (src/graphRead.cpp:2-26, instantiated at :47-51), compiled unchanged
// from its sources by oracle/Makefile.  TEST INFRASTRUCTURE ONLY.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>

template <typename T>
void readGraph(std::string filePath, T *&offset, T *&index, T &numVertices, T &numEdges);

// Reads <base>.info (the reference appends the suffix itself) and copies the
// arrays into caller buffers of at least cap_off / cap_ind entries.  Returns
// the vertex count, or -1 if a buffer is too small.
extern "C" int64_t ref_read_info(const char *base, int64_t *off_out, int64_t cap_off,
                                 int64_t *ind_out, int64_t cap_ind, int64_t *nnz_out)
{
    int64_t *off = nullptr, *ind = nullptr, nv = 0, ne = 0;
    readGraph<int64_t>(std::string(base), off, ind, nv, ne);
    int64_t rc = nv;
    if (nv + 1 > cap_off || ne > cap_ind) {
        rc = -1;
    } else {
        std::memcpy(off_out, off, sizeof(int64_t) * (size_t)(nv + 1));
        std::memcpy(ind_out, ind, sizeof(int64_t) * (size_t)ne);
        *nnz_out = ne;
    }
    delete[] off;
    delete[] ind;
    return rc;
}
