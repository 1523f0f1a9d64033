"""The C ABI library loads and exports every declared symbol; host-only
argument checks.  CPU only (no compute call needs a GPU here)."""
import ctypes
import os
import re

import pytest

from gputrianglecounting_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(gtc_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    decl = declared_functions()
    assert len(decl) >= 10
    for name in decl:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(_lib.exported_names()) <= set(decl) | {"gtc_status_string"}


def test_status_strings():
    lib = _lib.load()
    assert lib.gtc_status_string(0) == b"ok"
    assert lib.gtc_status_string(2) == b"invalid CSR"
    assert lib.gtc_status_string(99) == b"unknown status"


def test_workspace_size_host_only():
    lib = _lib.load()
    out = ctypes.c_size_t(0)
    assert lib.gtc_workspace_size(1000, 20000, 32, 0, ctypes.byref(out)) == 0
    plain = out.value
    assert plain > 20000 * 4
    assert lib.gtc_workspace_size(1000, 20000, 64, 1, ctypes.byref(out)) == 0
    assert out.value < plain + 8 * 1000 + 4096
    assert lib.gtc_workspace_size(1000, 20000, 16, 0, ctypes.byref(out)) == 1
    assert lib.gtc_workspace_size(-1, 0, 32, 0, ctypes.byref(out)) == 1
    assert lib.gtc_workspace_size(10, 0, 32, 7, ctypes.byref(out)) == 1
    assert lib.gtc_workspace_size(10, 1 << 33, 32, 0, ctypes.byref(out)) == 1
    assert lib.gtc_workspace_size(1 << 32, 10, 64, 0, ctypes.byref(out)) == 6


def test_launch_plan_host_only():
    """Label choice and kernel count per configuration, without a device."""
    from gputrianglecounting_b200 import api
    assert api.launch_plan(1 << 20, 12 << 20) == {"launches": 6, "labels": "vertex-id"}
    assert api.launch_plan(1 << 20, 30 << 20) == {"launches": 11, "labels": "degree-rank"}
    assert api.launch_plan(1 << 20, 30 << 20, mode="oriented")["launches"] == 10
    assert api.launch_plan(1000, 1000, tuning={"labels": 2})["labels"] == "degree-rank"
    assert api.launch_plan(1000, 90000, tuning={"labels": 1}) == {"launches": 5,
                                                                   "labels": "vertex-id"}
    with pytest.raises(_lib.GTCError):
        api.launch_plan(1000, 1000, tuning={"labels": 3})


def test_invalid_arguments_rejected_before_any_device_work():
    lib = _lib.load()
    # null offsets / workspace
    assert lib.gtc_count(None, 32, None, 10, 0, 0, None, None, None, None, None, 0, None) == 1
    # oriented mode with per-vertex outputs requested
    fake = ctypes.c_void_p(256)
    assert lib.gtc_count(fake, 32, fake, 10, 4, 1, fake, None, None, None, fake, 1 << 20,
                         None) == 1
    # misaligned workspace
    assert lib.gtc_count(fake, 32, fake, 10, 4, 0, None, None, None, None,
                         ctypes.c_void_p(257), 1 << 20, None) == 1
    # workspace too small
    assert lib.gtc_count(fake, 32, fake, 10, 4, 0, None, None, None, None, fake, 16, None) == 3
    # bad tuning
    bad = _lib.Tuning(group=12)
    assert lib.gtc_count_tuned(fake, 32, fake, 10, 4, 0, None, None, None, None, fake, 1 << 20,
                               None, ctypes.byref(bad)) == 1
    bad = _lib.Tuning(region=3)
    assert lib.gtc_count_tuned(fake, 32, fake, 10, 4, 0, None, None, None, None, fake, 1 << 20,
                               None, ctypes.byref(bad)) == 1
    bad = _lib.Tuning(labels=5)
    assert lib.gtc_count_tuned(fake, 32, fake, 10, 4, 0, None, None, None, None, fake, 1 << 20,
                               None, ctypes.byref(bad)) == 1
    # item_len above 32768 could carry a 16-bit shared hit counter into its
    # neighbour, and it must be a power of two; rejected (host-only check,
    # also in the launch plan)
    bad = _lib.Tuning(item_len=65536)
    assert lib.gtc_count_tuned(fake, 32, fake, 10, 4, 0, None, None, None, None, fake, 1 << 20,
                               None, ctypes.byref(bad)) == 1
    from gputrianglecounting_b200 import api
    assert api.launch_plan(1000, 90000, tuning={"item_len": 32768})["launches"] > 0
    for bad_len in (65536, 65535, 48, 100):
        with pytest.raises(_lib.GTCError):
            api.launch_plan(1000, 90000, tuning={"item_len": bad_len})
    # the merge form of the group kernel needs vertex-id labels: rejected with
    # rank labels, implies vertex ids with automatic labels
    for bad_tun in ({"rows": 3}, {"rows": -1}, {"rows": 2, "labels": 2}):
        with pytest.raises(_lib.GTCError):
            api.launch_plan(1000, 90000, tuning=bad_tun)
    assert api.launch_plan(1 << 20, 30 << 20, tuning={"rows": 2})["labels"] == "vertex-id"
    assert api.launch_plan(1 << 20, 30 << 20, tuning={"rows": 1})["labels"] == "degree-rank"
    # status query needs a workspace
    assert lib.gtc_count_status(None, 256, None, None) == 1
    assert lib.gtc_count_status(fake, 2, None, None) == 1
    # validator: misaligned workspace
    reason = ctypes.c_int32(-1)
    assert lib.gtc_validate_csr(fake, 32, fake, 10, 4, ctypes.c_void_p(264), 1 << 10,
                                ctypes.byref(reason), None) == 1
    assert lib.gtc_count_subset(None, 32, None, None, -1, None, None) == 1
    assert lib.gtc_count_subset(None, 32, None, None, 0, None, None) == 0


def test_compat_rejects_unsupported_block_size_without_launch():
    lib = _lib.load()
    lib.gtc_kernelCall_i64(10, 100, 5, None, None, None, 1, 100, 0)
    assert lib.gtc_compat_last_status() == 1
    lib.gtc_kernelCall_vertex_i32(10, 48, 5, None, None, None, None, 1, 48, 0)
    assert lib.gtc_compat_last_status() == 1


def test_package_fails_loudly_without_library(tmp_path):
    with pytest.raises(RuntimeError, match="not built"):
        saved = _lib._lib
        try:
            _lib._lib = None
            _lib.load(str(tmp_path / "missing.so"))
        finally:
            _lib._lib = saved


def test_reference_style_caller_compiles_and_links(tmp_path):
    """A caller written like the reference's host run path compiles against
    include/gtc_b200_kernelcall.hpp and links libgtc_b200.so (no GPU call)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "kernelcall_user"
    cmd = ["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "kernelcall_user.cpp"),
           "-L", lib_dir, "-lgtc_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    assert subprocess.run([str(exe)], capture_output=True).returncode == 0
