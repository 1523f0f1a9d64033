"""Host API of the B200 triangle counter (Python over the C ABI).

Mirrors the reference's operator surface for the per-vertex count:

* :func:`kernelCall` -- the reference host dispatcher
  (src/clusteringCount.cu:361-467) with its argument list and meaning:
  device CSR in, ``out[v] = r(v) = 2 t(v)`` out, tuning arguments as hints.
* :func:`count_triangles` / :class:`TriangleCounter` -- the native entry point
  (int32 or int64 offsets, int32 ids) returning r, t, lcc and the global count
  (T, the dest<src oriented sum 3T and the plain sum 6T), on a caller stream.
* :func:`count_subset`, :func:`validate_csr`.

Device memory and streams come from torch; every count runs in the CUDA
kernels of libgtc_b200.so.  There is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import GTCError, MODE_ORIENTED, MODE_PLAIN, check

__all__ = [
    "TriangleCounter", "TriangleCounts", "count_triangles", "count_subset",
    "validate_csr", "kernelCall", "GTCError",
]

_MODES = {"plain": MODE_PLAIN, "oriented": MODE_ORIENTED}


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_handle(stream) -> int | None:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream or None


def _check_csr_tensors(off: torch.Tensor, ind: torch.Tensor) -> int:
    if not (off.is_cuda and ind.is_cuda):
        raise ValueError("off and ind must be CUDA tensors (there is no host path)")
    if off.device != ind.device:
        raise ValueError("off and ind must be on the same device")
    if off.dtype not in (torch.int32, torch.int64):
        raise TypeError("off must be int32 or int64")
    if ind.dtype != torch.int32:
        raise TypeError("ind must be int32")
    if off.dim() != 1 or ind.dim() != 1 or not off.is_contiguous() or not ind.is_contiguous():
        raise ValueError("off and ind must be contiguous 1-D tensors")
    if off.numel() < 1:
        raise ValueError("off must hold n+1 >= 1 offsets")
    return 32 if off.dtype == torch.int32 else 64


def _alloc_workspace(nbytes: int, device) -> torch.Tensor:
    """A device workspace of at least nbytes (256-byte aligned: torch's
    caching allocator hands out 512-byte aligned blocks).  An allocation
    failure surfaces as GTCError(GTC_ERR_OUT_OF_MEMORY); the caller keeps no
    partial state."""
    try:
        return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
    except torch.cuda.OutOfMemoryError as e:
        raise GTCError(_lib.GTC_ERR_OUT_OF_MEMORY, f"workspace of {nbytes} bytes") from e


def _check_workspace_status(ws: torch.Tensor, stream) -> None:
    bits = ctypes.c_uint32(0)
    check(_lib.load().gtc_count_status(ws.data_ptr(), ws.numel(), _stream_handle(stream),
                                       ctypes.byref(bits)), "gtc_count_status")


@dataclass
class TriangleCounts:
    """Outputs of one count (device tensors; scalars read on demand)."""

    r: torch.Tensor | None          # int64[n]  = 2 t(v) (reference out[v])
    t: torch.Tensor | None          # int64[n]  triangles through v
    lcc: torch.Tensor | None        # float64[n] local clustering coefficient
    global_counts: torch.Tensor     # int64[3]  {T, 3T, 6T}

    @property
    def triangles(self) -> int:
        return int(self.global_counts[0].item())

    @property
    def oriented_sum(self) -> int:
        """dest<src oriented sum (README.md:6-10): 3T."""
        return int(self.global_counts[1].item())

    @property
    def total(self) -> int:
        """Sum of r, what src/gpurun.cu:40-49 prints as totalTriangleCount: 6T."""
        return int(self.global_counts[2].item())


class TriangleCounter:
    """Counts triangles on one CUDA device, reusing its workspace."""

    def __init__(self, device=None):
        _lib.load()
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self._ws: torch.Tensor | None = None

    def workspace_bytes(self, n: int, nnz: int, off_bits: int, mode: str = "plain") -> int:
        out = ctypes.c_size_t(0)
        check(_lib.load().gtc_workspace_size(n, nnz, off_bits, _MODES[mode], ctypes.byref(out)),
              "gtc_workspace_size")
        return int(out.value)

    def _workspace(self, nbytes: int) -> torch.Tensor:
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = None
            # 256-byte alignment: torch's caching allocator returns 512-aligned blocks
            self._ws = _alloc_workspace(nbytes, self.device)
        return self._ws

    def release(self) -> None:
        """Drop the cached workspace (it is re-allocated by the next count)."""
        self._ws = None

    def check_status(self, stream=None) -> None:
        """Device-side error report of the last count on this counter (waits
        for `stream`): raises GTCError(GTC_ERR_INVALID_CSR) if that count met
        a neighbour id outside [0, n), which the kernels skip instead of
        dereferencing."""
        if self._ws is not None:
            _check_workspace_status(self._ws, stream)

    def count(self, off: torch.Tensor, ind: torch.Tensor, mode: str = "plain",
              outputs=("r", "t", "lcc"), out: TriangleCounts | None = None,
              stream=None, tuning: dict | None = None) -> TriangleCounts:
        """Count triangles of a simple symmetric CSR (asynchronous on `stream`).

        mode "plain": per-vertex outputs (any of "r", "t", "lcc") + global.
        mode "oriented": global count only (the reference README's dest<src
        mode), no per-vertex bookkeeping.
        tuning: optional launch-shape overrides (keys of gtc_tuning: group,
        item_len, big_chunk, big_hash_max); they never change the result.
        """
        off_bits = _check_csr_tensors(off, ind)
        if mode not in _MODES:
            raise ValueError(f"mode must be one of {list(_MODES)}")
        n, nnz = off.numel() - 1, ind.numel()
        if out is None:
            dev = off.device
            want = set(outputs) if mode == "plain" else set()
            out = TriangleCounts(
                r=torch.empty(n, dtype=torch.int64, device=dev) if "r" in want else None,
                t=torch.empty(n, dtype=torch.int64, device=dev) if "t" in want else None,
                lcc=torch.empty(n, dtype=torch.float64, device=dev) if "lcc" in want else None,
                global_counts=torch.empty(3, dtype=torch.int64, device=dev),
            )
        ws_bytes = self.workspace_bytes(n, nnz, off_bits, mode)
        ws = self._workspace(ws_bytes)
        tun = None
        if tuning:
            tun = _lib.Tuning(**{k: int(v) for k, v in tuning.items()})
        st = _lib.load().gtc_count_tuned(
            off.data_ptr(), off_bits, ind.data_ptr() if nnz else None, n, nnz, _MODES[mode],
            _ptr(out.r), _ptr(out.t), _ptr(out.lcc), _ptr(out.global_counts),
            ws.data_ptr(), ws.numel(), _stream_handle(stream),
            ctypes.byref(tun) if tun is not None else None)
        check(st, "gtc_count")
        return out


def count_triangles(off: torch.Tensor, ind: torch.Tensor, mode: str = "plain",
                    outputs=("r", "t", "lcc"), stream=None) -> TriangleCounts:
    """One-shot count (allocates a workspace)."""
    return TriangleCounter(off.device).count(off, ind, mode=mode, outputs=outputs, stream=stream)


LABELS = {1: "vertex-id", 2: "degree-rank"}


def launch_plan(n: int, nnz: int, mode: str = "plain", tuning: dict | None = None) -> dict:
    """What a count of an (n, nnz) graph would run, host-only: kernel launches
    per count and the vertex labelling ("vertex-id" or "degree-rank")."""
    if mode not in _MODES:
        raise ValueError(f"mode must be one of {list(_MODES)}")
    tun = _lib.Tuning(**{k: int(v) for k, v in tuning.items()}) if tuning else None
    launches, labels = ctypes.c_int(0), ctypes.c_int(0)
    check(_lib.load().gtc_count_launches(n, nnz, _MODES[mode],
                                         ctypes.byref(tun) if tun is not None else None,
                                         ctypes.byref(launches), ctypes.byref(labels)),
          "gtc_count_launches")
    return {"launches": launches.value, "labels": LABELS[labels.value]}


def count_subset(off: torch.Tensor, ind: torch.Tensor, vertices: torch.Tensor,
                 stream=None) -> torch.Tensor:
    """r(v) for each listed vertex (the reference's vertex-list overload)."""
    off_bits = _check_csr_tensors(off, ind)
    if vertices.dtype != torch.int32 or not vertices.is_cuda:
        raise TypeError("vertices must be an int32 CUDA tensor")
    vertices = vertices.contiguous()
    out = torch.empty(vertices.numel(), dtype=torch.int64, device=off.device)
    check(_lib.load().gtc_count_subset(off.data_ptr(), off_bits, ind.data_ptr(),
                                       vertices.data_ptr(), vertices.numel(), out.data_ptr(),
                                       _stream_handle(stream)), "gtc_count_subset")
    return out


def validate_csr(off: torch.Tensor, ind: torch.Tensor, stream=None) -> tuple[int, str]:
    """Check the input contract on the device; returns (reason code, text)."""
    off_bits = _check_csr_tensors(off, ind)
    n, nnz = off.numel() - 1, ind.numel()
    lib = _lib.load()
    ws = torch.empty(lib.gtc_validate_workspace_size(n, nnz), dtype=torch.uint8,
                     device=off.device)
    reason = ctypes.c_int32(-1)
    check(lib.gtc_validate_csr(off.data_ptr(), off_bits, ind.data_ptr() if nnz else None, n, nnz,
                               ws.data_ptr(), ws.numel(), ctypes.byref(reason),
                               _stream_handle(stream)), "gtc_validate_csr")
    return reason.value, _lib.CSR_REASONS.get(reason.value, "unknown")


def kernelCall(numberBlocks: int, numberThreads: int, nv: int, d_off: torch.Tensor,
               d_ind: torch.Tensor, outPutTriangles: torch.Tensor, threads_per_block: int,
               number_blocks: int, shifter: int, vertex: torch.Tensor | None = None) -> None:
    """The reference's kernelCall<T> (src/clusteringCount.cu:361-467).

    T is taken from the tensors' dtype (int64 or int32, like the reference's
    two instantiations).  Without `vertex`: out[v] = r(v) for all nv vertices.
    With `vertex` (the vertex-list overload): out[k] = r(vertex[k]) for the nv
    listed vertices.  numberBlocks, threads_per_block, number_blocks and
    shifter are hints; an unsupported numberThreads launches nothing, as in the
    reference, and that or any other failure raises GTCError here.
    Asynchronous on the legacy default stream.
    """
    lib = _lib.load()
    dt = d_off.dtype
    if d_ind.dtype != dt or outPutTriangles.dtype != dt or (vertex is not None and vertex.dtype != dt):
        raise TypeError("all kernelCall tensors must share one integer dtype")
    if dt == torch.int64:
        fn = lib.gtc_kernelCall_i64 if vertex is None else lib.gtc_kernelCall_vertex_i64
    elif dt == torch.int32:
        fn = lib.gtc_kernelCall_i32 if vertex is None else lib.gtc_kernelCall_vertex_i32
    else:
        raise TypeError("kernelCall is instantiated for int32 and int64 only")
    if vertex is None:
        fn(numberBlocks, numberThreads, nv, d_off.data_ptr(), d_ind.data_ptr(),
           outPutTriangles.data_ptr(), threads_per_block, number_blocks, shifter)
    else:
        fn(numberBlocks, numberThreads, nv, vertex.data_ptr(), d_off.data_ptr(),
           d_ind.data_ptr(), outPutTriangles.data_ptr(), threads_per_block, number_blocks,
           shifter)
    check(lib.gtc_compat_last_status(), "kernelCall")


# ------------------------------------------------------------------ batched

@dataclass
class BatchCSR:
    """Many graphs in one concatenated CSR (device tensors).

    vstart[G+1] int64 vertex starts, off[N+1] int64 offsets into the
    concatenated adjacency, ind[NNZ] int32 graph-local neighbour ids.
    """

    vstart: torch.Tensor
    off: torch.Tensor
    ind: torch.Tensor

    @property
    def num_graphs(self) -> int:
        return int(self.vstart.numel()) - 1

    @property
    def total_n(self) -> int:
        return int(self.off.numel()) - 1

    @property
    def total_nnz(self) -> int:
        return int(self.ind.numel())

    def graph(self, g: int):
        """Graph g alone as a CSRGraph (offsets rebased to 0, same device)."""
        from .graphs import CSRGraph
        v0, v1 = int(self.vstart[g]), int(self.vstart[g + 1])
        off = self.off[v0:v1 + 1]
        e0, e1 = int(off[0]), int(off[-1])
        return CSRGraph((off - e0).contiguous(), self.ind[e0:e1].contiguous(), f"g{g}")


def batch_workspace_bytes(num_graphs: int, total_n: int, total_nnz: int) -> int:
    """Device workspace of one gtc_count_batch call (host-only query)."""
    out = ctypes.c_size_t(0)
    check(_lib.load().gtc_batch_workspace_size(num_graphs, total_n, total_nnz,
                                               ctypes.byref(out)), "gtc_batch_workspace_size")
    return int(out.value)


@dataclass
class BatchCounts:
    r: torch.Tensor | None          # int64[N] over the concatenated vertex space
    t: torch.Tensor | None
    lcc: torch.Tensor | None
    graph_T: torch.Tensor | None    # int64[G]


class BatchCounter:
    """Counts a whole batch of graphs in one pipeline run (one device)."""

    def __init__(self, device=None):
        _lib.load()
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self._ws: torch.Tensor | None = None
        self._pack_scratch: torch.Tensor | None = None
        self._pack_staging: torch.Tensor | None = None

    def workspace_bytes(self, num_graphs: int, total_n: int, total_nnz: int) -> int:
        return batch_workspace_bytes(num_graphs, total_n, total_nnz)

    def reserve(self, num_graphs: int, total_n: int, total_nnz: int) -> None:
        """Allocate the workspace up front (e.g. before a CUDA-graph capture)."""
        need = self.workspace_bytes(num_graphs, total_n, total_nnz)
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = _alloc_workspace(need, self.device)

    def release(self) -> None:
        """Drop the cached workspace and pack buffers."""
        self._ws = None
        self._pack_scratch = None
        self._pack_staging = None

    def check_status(self, stream=None) -> None:
        """As TriangleCounter.check_status, for the last batch counted here
        (a local id outside its graph's [0, n_g) raises GTC_ERR_INVALID_CSR)."""
        if self._ws is not None:
            _check_workspace_status(self._ws, stream)

    def alloc_outputs(self, batch: BatchCSR, outputs=("r", "lcc", "graph_T")) -> BatchCounts:
        dev, n, G = self.device, batch.total_n, batch.num_graphs
        return BatchCounts(
            r=torch.empty(n, dtype=torch.int64, device=dev) if "r" in outputs else None,
            t=torch.empty(n, dtype=torch.int64, device=dev) if "t" in outputs else None,
            lcc=torch.empty(n, dtype=torch.float64, device=dev) if "lcc" in outputs else None,
            graph_T=torch.empty(G, dtype=torch.int64, device=dev) if "graph_T" in outputs else None)

    def count(self, batch: BatchCSR, outputs=("r", "lcc", "graph_T"), out: BatchCounts | None = None,
              tuning: dict | None = None, stream=None) -> BatchCounts:
        G, n, nnz = batch.num_graphs, batch.total_n, batch.total_nnz
        self.reserve(G, n, nnz)
        if out is None:
            out = self.alloc_outputs(batch, outputs)
        tun = _lib.Tuning(**{k: int(v) for k, v in tuning.items()}) if tuning else None
        check(_lib.load().gtc_count_batch(
            G, batch.vstart.data_ptr(), batch.off.data_ptr(),
            batch.ind.data_ptr() if nnz else None, n, nnz, _ptr(out.r), _ptr(out.t),
            _ptr(out.lcc), _ptr(out.graph_T), self._ws.data_ptr(), self._ws.numel(),
            ctypes.byref(tun) if tun is not None else None, _stream_handle(stream)),
            "gtc_count_batch")
        return out

    def pack(self, graphs, stream=None) -> BatchCSR:
        """Concatenate separate device-resident graphs (int64 off, int32 ind)."""
        G = len(graphs)
        lib = _lib.load()
        need = int(lib.gtc_batch_pack_scratch_bytes(G))
        if self._pack_scratch is None or self._pack_scratch.numel() < need:
            self._pack_scratch = torch.empty(need, dtype=torch.uint8, device=self.device)
            self._pack_staging = torch.empty(need, dtype=torch.uint8).pin_memory()
        else:
            # the staging buffer may still feed an earlier copy
            torch.cuda.current_stream(self.device).synchronize()
        offs = (ctypes.c_void_p * max(G, 1))(*[g.off.data_ptr() for g in graphs])
        inds = (ctypes.c_void_p * max(G, 1))(*[g.ind.data_ptr() for g in graphs])
        ns = (ctypes.c_int64 * max(G, 1))(*[g.n for g in graphs])
        nnzs = (ctypes.c_int64 * max(G, 1))(*[g.nnz for g in graphs])
        total_n, total_nnz = sum(g.n for g in graphs), sum(g.nnz for g in graphs)
        vstart = torch.empty(G + 1, dtype=torch.int64, device=self.device)
        off = torch.empty(total_n + 1, dtype=torch.int64, device=self.device)
        ind = torch.empty(max(total_nnz, 1), dtype=torch.int32, device=self.device)[:total_nnz]
        check(lib.gtc_batch_pack(G, offs, inds, ns, nnzs, vstart.data_ptr(), off.data_ptr(),
                                 ind.data_ptr() if total_nnz else None,
                                 self._pack_scratch.data_ptr(), self._pack_scratch.numel(),
                                 self._pack_staging.data_ptr(), _stream_handle(stream)),
              "gtc_batch_pack")
        return BatchCSR(vstart, off, ind)
