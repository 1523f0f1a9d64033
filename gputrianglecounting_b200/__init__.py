"""B200-native per-vertex triangle counter (drop-in for the
count_all_trianglesGPU / kernelCall operator of ogreen/GpuTriangleCounting).

Public API: :mod:`gputrianglecounting_b200.api` (counting, validation,
reference-compatible kernelCall), :mod:`gputrianglecounting_b200.graphs`
(seeded synthetic inputs).  The native library is libgtc_b200.so, built from
csrc/ for sm_100a.
"""
from . import api, graphs  # noqa: F401

__all__ = ["api", "graphs"]
