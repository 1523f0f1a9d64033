"""ctypes binding of libgtc_b200.so (the C ABI declared in include/gtc_b200.h).

The shared library is built in-tree (gputrianglecounting_b200/libgtc_b200.so)
by `python -c "import __graft_entry__; __graft_entry__.build()"` or
`make -C gputrianglecounting_b200/csrc`.  There is no fallback: if the library
is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_uint, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgtc_b200.so")

# gtc_status values
GTC_OK = 0
GTC_ERR_INVALID_CSR = 2
GTC_ERR_OUT_OF_MEMORY = 5
STATUS_NAMES = {
    0: "GTC_OK", 1: "GTC_ERR_INVALID_ARGUMENT", 2: "GTC_ERR_INVALID_CSR",
    3: "GTC_ERR_WORKSPACE_TOO_SMALL", 4: "GTC_ERR_CUDA", 5: "GTC_ERR_OUT_OF_MEMORY",
    6: "GTC_ERR_UNSUPPORTED", 7: "GTC_ERR_TIMEOUT", 8: "GTC_ERR_CAPACITY", 9: "GTC_ERR_BUSY",
}
MODE_PLAIN, MODE_ORIENTED = 0, 1
CSR_REASONS = {0: "ok", 1: "bad offsets", 2: "index out of range", 3: "self-loop",
               4: "row not strictly ascending", 5: "not symmetric"}

P = c_void_p
_SIGNATURES = {
    "gtc_status_string": (c_char_p, [c_int]),
    "gtc_device_info": (c_int, [P, P]),
    "gtc_workspace_size": (c_int, [c_int64, c_int64, c_int, c_int, P]),
    "gtc_count": (c_int, [P, c_int, P, c_int64, c_int64, c_int, P, P, P, P, P, c_size_t, P]),
    "gtc_count_tuned": (c_int, [P, c_int, P, c_int64, c_int64, c_int, P, P, P, P, P, c_size_t, P,
                                P]),
    "gtc_count_launches": (c_int, [c_int64, c_int64, c_int, P, P, P]),
    "gtc_count_status": (c_int, [P, c_size_t, P, P]),
    "gtc_count_phase_times": (c_int, [P, c_int, P, c_int64, c_int64, P, c_size_t, P, P]),
    "gtc_count_noalloc": (c_int, [P, c_int, P, c_int64, c_int64, c_int, P, P, P, P, P]),
    "gtc_batch_workspace_size": (c_int, [c_int64, c_int64, c_int64, P]),
    "gtc_count_batch": (c_int, [c_int64, P, P, P, c_int64, c_int64, P, P, P, P, P, c_size_t, P,
                                P]),
    "gtc_batch_pack_scratch_bytes": (c_size_t, [c_int64]),
    "gtc_batch_pack": (c_int, [c_int64, P, P, P, P, P, P, P, P, c_size_t, P, P]),
    "gtc_count_subset": (c_int, [P, c_int, P, P, c_int64, P, P]),
    "gtc_validate_workspace_size": (c_size_t, [c_int64, c_int64]),
    "gtc_validate_csr": (c_int, [P, c_int, P, c_int64, c_int64, P, c_size_t, P, P]),
    "gtc_kernelCall_i64": (None, [c_uint, c_uint, c_int64, P, P, P, c_int64, c_int64, c_int64]),
    "gtc_kernelCall_i32": (None, [c_uint, c_uint, c_int32, P, P, P, c_int32, c_int32, c_int32]),
    "gtc_kernelCall_vertex_i64": (None, [c_uint, c_uint, c_int64, P, P, P, P, c_int64, c_int64,
                                         c_int64]),
    "gtc_kernelCall_vertex_i32": (None, [c_uint, c_uint, c_int32, P, P, P, P, c_int32, c_int32,
                                         c_int32]),
    "gtc_compat_last_status": (c_int, []),
    "gtc_compat_release": (c_int, []),
}



class Tuning(ctypes.Structure):
    """gtc_tuning (0 = library choice)."""
    _fields_ = [("group", c_int), ("item_len", c_int), ("big_chunk", c_int),
                ("big_hash_max", c_int), ("labels", c_int), ("region", c_int),
                ("rows", c_int)]


_lib = None


class GTCError(RuntimeError):
    """A C-ABI call returned a non-OK gtc_status."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{what}: {name}" if what else name)


def load(path: str | None = None) -> ctypes.CDLL:
    """Load the native library (once).  Raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is not built; run `make -C gputrianglecounting_b200/csrc` "
            "(the CUDA path has no fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "") -> None:
    if status != GTC_OK:
        raise GTCError(status, what)


def exported_names() -> list[str]:
    return list(_SIGNATURES)
