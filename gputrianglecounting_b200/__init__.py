"""B200-native per-vertex triangle counter (drop-in for the
count_all_trianglesGPU / kernelCall operator of ogreen/GpuTriangleCounting).

Public API: :mod:`.api` (counting, batched counting, validation,
reference-compatible kernelCall), :mod:`.serve` (continuous-batching server),
:mod:`.autotune` (launch-shape tuner), :mod:`.formats` (`.info` and METIS
files), :mod:`.graphs` (seeded synthetic inputs).  The native library is libgtc_b200.so, built from
csrc/ for sm_100a.
"""
from . import api, autotune, formats, graphs, serve  # noqa: F401

__all__ = ["api", "autotune", "formats", "graphs", "serve"]
