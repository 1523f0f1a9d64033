"""Loader for the CPU oracle and the reference built from its sources.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, never by the product package.

* libtc_oracle.so  -- oracle/tc_oracle.c, a C restatement of the reference's
  CPU count (src/clusteringCount.cpp:2-155) with the LCC and global formulas.
* _ref/libref_cpu.so -- the reference's own src/clusteringCount.cpp compiled
  unchanged (oracle/Makefile target `ref`) behind oracle/ref_cpu_shim.cpp.
* _ref/libref_gpu.so -- the reference's own src/clusteringCount.cu compiled for
  sm_100a behind oracle/ref_gpu_shim.cu (GPU tests only, tpi = 1).
* _ref/libref_formats.so -- the reference's METIS converter
  (src/csrdatacreate.cpp) and `.info` reader (src/graphRead.cpp) behind
  oracle/ref_formats_shim.cpp and oracle/ref_info_shim.cpp (format tests).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_int, c_int64, c_uint, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libtc_oracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

_cache: dict[str, ctypes.CDLL] = {}


def _load(path: str, sigs: dict) -> ctypes.CDLL:
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not built (make -C oracle oracle ref)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _cache[path] = lib
    return lib


def oracle_lib() -> ctypes.CDLL:
    P = c_void_p
    return _load(ORACLE_SO, {
        "oracle_tri_ne": (c_int64, [c_int64, P, P, P]),
        "oracle_per_vertex": (c_int64, [c_int64, P, P, P, P, P, c_int]),
        "oracle_oriented_sum": (c_int64, [c_int64, P, P, c_int]),
        "oracle_subset": (None, [c_int64, P, P, P, P, c_int]),
        "oracle_max_threads": (c_int, []),
    })


def ref_cpu_available() -> bool:
    return os.path.exists(REF_CPU_SO)


def ref_cpu_lib() -> ctypes.CDLL:
    P = c_void_p
    return _load(REF_CPU_SO, {
        "ref_cpu_tri_ne_i64": (c_int64, [c_int64, P, P, P]),
        "ref_cpu_tri_ne_i32": (c_int64, [ctypes.c_int32, P, P, P]),
        "ref_cpu_rows_omp_i64": (c_int64, [c_int64, P, P, P, c_int64, P, P, c_int]),
        "ref_cpu_units_timed_i32": (c_int64, [ctypes.c_int32, P, P, P, P, P, c_int64, P, P, P,
                                              c_int]),
        "ref_cpu_max_threads": (c_int, []),
    })


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def ref_gpu_lib() -> ctypes.CDLL:
    P = c_void_p
    return _load(REF_GPU_SO, {
        "ref_gpu_count_i64": (c_int, [c_uint, c_uint, c_int64, P, P, P]),
    })


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(c_void_p)


# ----------------------------------------------------------------- oracle

def per_vertex(off, ind, threads: int = 0):
    """(r, t, lcc, sum_r) from the C restatement."""
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int32)
    n = off.shape[0] - 1
    r = np.zeros(n, np.int64)
    t = np.zeros(n, np.int64)
    lcc = np.zeros(n, np.float64)
    total = oracle_lib().oracle_per_vertex(n, po, pi, r.ctypes.data_as(c_void_p),
                                           t.ctypes.data_as(c_void_p),
                                           lcc.ctypes.data_as(c_void_p), threads)
    return r, t, lcc, int(total)


def tri_ne(off, ind):
    """Per directed edge |N(src) ∩ N(dst)|, CSR order, and its sum."""
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int32)
    out = np.zeros(ind.shape[0], np.int64)
    total = oracle_lib().oracle_tri_ne(off.shape[0] - 1, po, pi, out.ctypes.data_as(c_void_p))
    return out, int(total)


def oriented_sum(off, ind, threads: int = 0) -> int:
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int32)
    return int(oracle_lib().oracle_oriented_sum(off.shape[0] - 1, po, pi, threads))


def subset(off, ind, vertices, threads: int = 0):
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int32)
    vertices, pv = _arr(vertices, np.int32)
    out = np.zeros(vertices.shape[0], np.int64)
    oracle_lib().oracle_subset(vertices.shape[0], pv, po, pi, out.ctypes.data_as(c_void_p), threads)
    return out


def lcc_formula(r: np.ndarray, deg: np.ndarray) -> np.ndarray:
    """lcc = r / (d (d-1)) with d(d-1) formed in int64, 0 when d < 2."""
    r = np.asarray(r, np.int64)
    deg = np.asarray(deg, np.int64)
    pairs = deg * (deg - 1)
    out = np.zeros(r.shape[0], np.float64)
    ok = deg >= 2
    out[ok] = r[ok].astype(np.float64) / pairs[ok].astype(np.float64)
    return out


# -------------------------------------------------------------- reference

def ref_tri_ne(off, ind):
    """The reference's own count_all_trianglesCPU<int64_t> (serial)."""
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int64)
    out = np.zeros(ind.shape[0], np.int64)
    total = ref_cpu_lib().ref_cpu_tri_ne_i64(off.shape[0] - 1, po, pi,
                                             out.ctypes.data_as(c_void_p))
    return out, int(total)


def ref_rows(off, ind, vertices=None, threads: int = 0):
    """The reference's vertex-list count, one vertex per call, OpenMP.

    Returns (r for every processed row (0 elsewhere), total over processed rows).
    """
    off, po = _arr(off, np.int64)
    ind, pi = _arr(ind, np.int64)
    n = off.shape[0] - 1
    tri = np.zeros(ind.shape[0], np.int64)
    r = np.zeros(n, np.int64)
    if vertices is None:
        total = ref_cpu_lib().ref_cpu_rows_omp_i64(n, po, pi, None, n, tri.ctypes.data_as(c_void_p),
                                                   r.ctypes.data_as(c_void_p), threads)
    else:
        vertices, pv = _arr(vertices, np.int64)
        total = ref_cpu_lib().ref_cpu_rows_omp_i64(n, po, pi, pv, vertices.shape[0],
                                                   tri.ctypes.data_as(c_void_p),
                                                   r.ctypes.data_as(c_void_p), threads)
    return r, int(total)


def ref_prepared(off, ind):
    """int64 copies of a CSR laid out for ref_rows_prepared (timed loops)."""
    return np.ascontiguousarray(off, np.int64), np.ascontiguousarray(ind, np.int64)


def ref_rows_prepared(off64, ind64, vertices64, tri, r, threads: int = 0) -> int:
    """ref_rows without conversions (arrays already int64, outputs preallocated)."""
    return int(ref_cpu_lib().ref_cpu_rows_omp_i64(
        off64.shape[0] - 1, off64.ctypes.data_as(c_void_p), ind64.ctypes.data_as(c_void_p),
        None if vertices64 is None else vertices64.ctypes.data_as(c_void_p),
        off64.shape[0] - 1 if vertices64 is None else vertices64.shape[0],
        tri.ctypes.data_as(c_void_p), r.ctypes.data_as(c_void_p), threads))


def ref_units_timed(off32, ind32, unit_rows, unit_off, units, threads: int = 0,
                    tri=None, r=None):
    """The reference's vertex-list count (int32 CSR) over the listed units of
    rows (unit u = unit_rows[unit_off[u]:unit_off[u+1]]), one unit per
    OpenMP task.  Returns (unit_ns int64[len(units)], total of triNE over the
    rows run).  tri and r (int64[nnz], int64[n]) may be passed preallocated;
    r[v] receives each run row's sum of triNE."""
    off32 = np.ascontiguousarray(off32, np.int32)
    ind32 = np.ascontiguousarray(ind32, np.int32)
    unit_rows = np.ascontiguousarray(unit_rows, np.int64)
    unit_off = np.ascontiguousarray(unit_off, np.int64)
    units = np.ascontiguousarray(units, np.int64)
    if tri is None:
        tri = np.zeros(ind32.shape[0], np.int64)
    if r is None:
        r = np.zeros(off32.shape[0] - 1, np.int64)
    ns = np.zeros(units.shape[0], np.int64)
    P = lambda a: a.ctypes.data_as(c_void_p)  # noqa: E731
    total = ref_cpu_lib().ref_cpu_units_timed_i32(
        off32.shape[0] - 1, P(off32), P(ind32), P(unit_rows), P(unit_off), P(units),
        units.shape[0], P(tri), P(r), P(ns), threads)
    return ns, int(total)


def ref_all_rows_i32(off32, ind32, threads: int = 0, chunk: int = 64):
    """r for every row through the timed form (units of `chunk` consecutive
    rows); returns (r, total)."""
    n = off32.shape[0] - 1
    rows = np.arange(n, dtype=np.int64)
    uoff = np.minimum(np.arange(0, n + chunk, chunk, dtype=np.int64), n)
    uoff = np.unique(uoff)
    r = np.zeros(n, np.int64)
    _, total = ref_units_timed(off32, ind32, rows, uoff, np.arange(uoff.shape[0] - 1), threads,
                               r=r)
    return r, total


def max_threads() -> int:
    return int(oracle_lib().oracle_max_threads())


# ---------------------------------------------------------------- formats

REF_FORMATS_SO = os.path.join(HERE, "_ref", "libref_formats.so")


def ref_formats_available() -> bool:
    return os.path.exists(REF_FORMATS_SO)


def ref_formats_lib() -> ctypes.CDLL:
    P = c_void_p
    return _load(REF_FORMATS_SO, {
        "ref_metis_to_info": (c_int64, [ctypes.c_char_p, ctypes.c_char_p, P]),
        "ref_read_info": (c_int64, [ctypes.c_char_p, P, c_int64, P, c_int64, P]),
    })


def ref_metis_to_info(metis_path: str, info_path: str) -> int:
    """The reference's own converter (src/csrdatacreate.cpp) writing .info."""
    nnz = ctypes.c_int64(0)
    return int(ref_formats_lib().ref_metis_to_info(metis_path.encode(), info_path.encode(),
                                                    ctypes.byref(nnz)))


def ref_read_info(base: str, cap_n: int, cap_nnz: int):
    """The reference's own .info reader (src/graphRead.cpp); reads base + '.info'."""
    off = np.zeros(cap_n + 1, np.int64)
    ind = np.zeros(max(cap_nnz, 1), np.int64)
    nnz = ctypes.c_int64(0)
    n = ref_formats_lib().ref_read_info(base.encode(), off.ctypes.data_as(c_void_p), cap_n + 1,
                                        ind.ctypes.data_as(c_void_p), cap_nnz, ctypes.byref(nnz))
    if n < 0:
        raise RuntimeError("buffers too small")
    return off[:n + 1], ind[:nnz.value]
