// ref_formats_shim.cpp -- extern "C" entry points over the reference's own
// METIS -> CSR converter (src/csrdatacreate.cpp: readGraph vector overload
// :3-47 and writeGraph :86-114).  That file holds templates only (no
// instantiations), so it is compiled into this translation unit from where it
// lies in the reference (oracle/Makefile passes its path).  TEST
// INFRASTRUCTURE ONLY: the format tests compare the product's writer/reader
// with the reference's byte for byte.
#include <cstdint>
#include <string>
#include <vector>

#include REF_CSRDATACREATE   // the reference's src/csrdatacreate.cpp

extern "C" int64_t ref_metis_to_info(const char *metis_path, const char *info_path,
                                     int64_t *nnz_out)
{
    std::vector<int64_t> off, ind;
    int64_t nv = 0, ne = 0;
    readGraph<int64_t>(std::string(metis_path), off, ind, nv, ne);
    writeGraph<int64_t>(std::string(info_path), off, ind);
    if (nnz_out) *nnz_out = (int64_t)ind.size();
    return (int64_t)off.size() - 1;
}
