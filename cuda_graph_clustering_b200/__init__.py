"""B200-native PBILS k-correlation clustering: Python mirror of the reference's solver interface.

The reference (oQaris/cuda_graph_clustering) exposes ``cc::SolveGpu``,
``cc::SolveNeighborhoodGpu`` and ``cc::SolveNeighborhoodWithManyLocalSearchesGpu`` over
``cc::Graph`` and ``cc::PbilsParams`` (include/cc_gpu.hpp:10-20, include/cc_pbils.hpp:26-59).  This
module keeps those names, argument meanings and errors (``RuntimeError`` with the reference's
message) over the C ABI of ``libccb.so`` (include/ccb.h).  Every compute call runs the hand-written
sm_100a kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import (CcbError, CcbParams, CcbResult, CcbKernelStats, CcbTuningEntry, LS_AUTO, LS_GLOBAL, LS_SHARED, LS_WIDE,
                      MAX_CLUSTERS, MAX_VERTICES_NARROW, MAX_VERTICES_WIDE, check, lib)

__all__ = ["Graph", "PbilsParams", "PbilsResult", "SolveGpu", "SolveNeighborhoodGpu",
           "SolveNeighborhoodWithManyLocalSearchesGpu", "DeviceGraph", "Solver", "Batch", "Server", "CcbError",
           "set_tuning", "get_tuning", "load_tuning", "LS_AUTO", "LS_GLOBAL",
           "LS_SHARED", "LS_WIDE", "MAX_CLUSTERS", "kMaxClusters"]

kMaxClusters = MAX_CLUSTERS  # include/cc_gpu.hpp:10


def words_per_row(n: int) -> int:
    """cc::Graph's row length: max(1, ceil(n / 32)) words (src/cc_graph.cpp:149-153)."""
    return 1 if n == 0 else (n + 31) // 32


class Graph:
    """Undirected, unweighted, loop-free graph as the reference's bitset (include/cc_graph.hpp:15-59)."""

    def __init__(self, n: int = 0, bits: np.ndarray | None = None, edges: int | None = None):
        self.n = int(n)
        w = words_per_row(self.n)
        if bits is None:
            bits = np.zeros((self.n, w), np.uint32)
        self.bits = np.ascontiguousarray(bits, dtype=np.uint32).reshape(self.n, -1 if self.n else w)
        if self.bits.shape[1] < (self.n + 31) // 32:
            raise ValueError("rows shorter than ceil(n / 32) words")
        self.edges = int(edges) if edges is not None else int(sum(int(x).bit_count() for x in self.bits.ravel())) // 2

    def Size(self) -> int:
        return self.n

    def WordsPerRow(self) -> int:
        return self.bits.shape[1]

    def EdgeCount(self) -> int:
        return self.edges

    def IsJoined(self, i: int, j: int) -> bool:
        return bool((int(self.bits[i, j // 32]) >> (j % 32)) & 1)

    def AddEdge(self, i: int, j: int) -> None:
        if i == j or self.IsJoined(i, j):
            return
        self.bits[i, j // 32] |= np.uint32(1 << (j % 32))
        self.bits[j, i // 32] |= np.uint32(1 << (i % 32))
        self.edges += 1

    def Density(self) -> float:
        pairs = self.n * (self.n - 1) / 2
        return self.edges / pairs if pairs > 0 else 0.0

    @staticmethod
    def ErdosRenyi(n: int, density: float, seed: int) -> "Graph":
        """Graph::ErdosRenyi (src/cc_graph.cpp:168-177), generated by libccb on the host."""
        w = words_per_row(n)
        bits = np.zeros((max(n, 1), w), np.uint32)
        edges = lib().ccb_generate_erdos_renyi(n, density, seed, bits.ctypes.data, w)
        return Graph(n, bits[:n], edges)

    @staticmethod
    def Planted(n: int, parts: int, p_in: float, p_out: float, flip: float, seed: int,
                shuffle_split: bool = False) -> tuple["Graph", np.ndarray]:
        """Seeded planted partition (this project's generator; no counterpart in the reference)."""
        w = words_per_row(n)
        bits = np.zeros((max(n, 1), w), np.uint32)
        comm = np.zeros(max(n, 1), np.int32)
        edges = lib().ccb_generate_planted(n, parts, int(shuffle_split), p_in, p_out, flip, seed, bits.ctypes.data,
                                           w, comm.ctypes.data)
        return Graph(n, bits[:n], edges), comm[:n]


@dataclass
class PbilsParams:
    """cc::PbilsParams (include/cc_pbils.hpp:26-49) with its defaults."""

    k: int = 2
    population: int = 128
    tournament: int = 5
    iterations: int = 100
    early_stop: int = 6
    perturbation: float = 0.4
    gww: float = 0.1
    threads: int = 1
    seed: int = 1
    time_limit_sec: float = 0.0
    verbose: bool = False
    ls_kernel: int = LS_AUTO

    def to_c(self) -> CcbParams:
        return CcbParams(self.k, self.population, self.tournament, self.iterations, self.early_stop,
                         self.perturbation, self.gww, self.threads, self.seed, self.time_limit_sec,
                         int(bool(self.verbose)), self.ls_kernel)


@dataclass
class PbilsResult:
    """cc::PbilsResult (include/cc_pbils.hpp:51-59)."""

    objective: int = -1
    labels: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    iterations_done: int = 0
    clusters_used: int = 0
    seconds: float = 0.0
    local_searches: int = 0
    accepted_moves: int = 0

    @staticmethod
    def from_c(r: CcbResult, labels: np.ndarray) -> "PbilsResult":
        return PbilsResult(int(r.objective), labels, int(r.iterations_done), int(r.clusters_used), float(r.seconds),
                           int(r.local_searches), int(r.accepted_moves))


def _run(fn, graph: Graph, params: PbilsParams, *extra) -> PbilsResult:
    labels = np.zeros(max(graph.n, 1), np.int32)
    res = CcbResult()
    p = params.to_c()
    status = fn(graph.bits.ctypes.data if graph.n else None, graph.n, graph.WordsPerRow(), graph.edges, C.byref(p),
                *extra, labels.ctypes.data, C.byref(res))
    check(status)
    return PbilsResult.from_c(res, labels[: graph.n])


def SolveGpu(graph: Graph, params: PbilsParams) -> PbilsResult:
    """cc::SolveGpu (cuda/cc_pbils_gpu.cu:441-454)."""
    return _run(lib().ccb_pbils_solve, graph, params)


def SolveNeighborhoodGpu(graph: Graph, params: PbilsParams) -> PbilsResult:
    """cc::SolveNeighborhoodGpu (cuda/cc_pbils_gpu.cu:456-458)."""
    return _run(lib().ccb_neighborhood_solve, graph, params, 0)


def SolveNeighborhoodWithManyLocalSearchesGpu(graph: Graph, params: PbilsParams) -> PbilsResult:
    """cc::SolveNeighborhoodWithManyLocalSearchesGpu (cuda/cc_pbils_gpu.cu:460-462)."""
    return _run(lib().ccb_neighborhood_solve, graph, params, 1)


class DeviceGraph:
    """A graph kept on the device across solves (ccb_graph_upload / ccb_graph_from_device)."""

    def __init__(self, graph: Graph | None = None, stream: int = 0, device_ptr: int | None = None, n: int = 0,
                 words: int = 0, edges: int = 0):
        h = C.c_void_p()
        if graph is not None:
            check(lib().ccb_graph_upload(graph.bits.ctypes.data if graph.n else None, graph.n, graph.WordsPerRow(),
                                         graph.edges, stream or None, C.byref(h)))
            self.n, self.edges = graph.n, graph.edges
        else:
            check(lib().ccb_graph_from_device(device_ptr, n, words, edges, stream or None, C.byref(h)))
            self.n, self.edges = n, edges
        self.handle = h

    @classmethod
    def _wrap(cls, handle: C.c_void_p) -> "DeviceGraph":
        g = cls.__new__(cls)
        g.handle = handle
        n = C.c_uint32()
        e = C.c_uint64()
        check(lib().ccb_graph_size(handle, C.byref(n), C.byref(e)))
        g.n, g.edges = int(n.value), int(e.value)
        return g

    @classmethod
    def erdos_renyi(cls, n: int, density: float, seed: int, stream: int = 0) -> "DeviceGraph":
        """Graph::ErdosRenyi generated on the device (same bits as the host generator)."""
        h = C.c_void_p()
        check(lib().ccb_graph_generate_erdos_renyi(n, density, seed, stream or None, C.byref(h)))
        return cls._wrap(h)

    @classmethod
    def planted(cls, n: int, parts: int, p_in: float, p_out: float, flip: float, seed: int,
                shuffle_split: bool = False, stream: int = 0) -> tuple["DeviceGraph", np.ndarray]:
        """The planted partition generated on the device (same bits as Graph.Planted)."""
        h = C.c_void_p()
        comm = np.zeros(max(n, 1), np.int32)
        check(lib().ccb_graph_generate_planted(n, parts, int(shuffle_split), p_in, p_out, flip, seed, stream or None,
                                               C.byref(h), comm.ctypes.data))
        return cls._wrap(h), comm[:n]

    @classmethod
    def load_tags(cls, path: str, similarity: str = "jaccard", threshold: float = 0.5, n: int = 0, seed: int = 1,
                  stream: int = 0) -> "DeviceGraph":
        """Graph::LoadTags (src/cc_graph.cpp:311-371) built on the device (ccb_graph_load_tags)."""
        h = C.c_void_p()
        check(lib().ccb_graph_load_tags(path.encode(), similarity.encode(), threshold, n, seed, stream or None,
                                        C.byref(h)))
        return cls._wrap(h)

    def download(self) -> Graph:
        w = words_per_row(self.n)
        bits = np.zeros((max(self.n, 1), w), np.uint32)
        check(lib().ccb_graph_download(self.handle, bits.ctypes.data, w))
        return Graph(self.n, bits[: self.n], self.edges)

    def close(self) -> None:
        if self.handle:
            lib().ccb_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REBUILD_KINDS = {"auto": 0, "popcount": 1, "tensor": 2}


class Solver:
    """Reusable buffers and kernel plan for (graph, k, population, ls_kernel) (ccb_solver_*)."""

    def __init__(self, graph: DeviceGraph, params: PbilsParams):
        h = C.c_void_p()
        p = params.to_c()
        check(lib().ccb_solver_create(graph.handle, C.byref(p), C.byref(h)))
        self.handle = h
        self.graph = graph
        self.n = graph.n

    def describe(self) -> str:
        return lib().ccb_solver_describe(self.handle).decode()

    def set_rebuild(self, kind: str) -> None:
        """How G = A*Z is rebuilt (ccb_solver_set_rebuild): "auto", "popcount" or "tensor" (int8 tcgen05)."""
        check(lib().ccb_solver_set_rebuild(self.handle, REBUILD_KINDS[kind]))

    def set_profiling(self, on: bool) -> None:
        check(lib().ccb_solver_set_profiling(self.handle, int(on)))

    def stats(self) -> CcbKernelStats:
        s = CcbKernelStats()
        check(lib().ccb_solver_stats(self.handle, C.byref(s)))
        return s

    def pbils(self, params: PbilsParams, stream: int = 0, want_labels: bool = True) -> PbilsResult:
        labels = np.zeros(max(self.n, 1), np.int32)
        res = CcbResult()
        p = params.to_c()
        check(lib().ccb_solver_pbils(self.handle, C.byref(p), stream or None,
                                     labels.ctypes.data if want_labels else None, C.byref(res)))
        return PbilsResult.from_c(res, labels[: self.n])

    def neighborhood(self, params: PbilsParams, local_search: bool, stream: int = 0) -> PbilsResult:
        labels = np.zeros(max(self.n, 1), np.int32)
        res = CcbResult()
        p = params.to_c()
        check(lib().ccb_solver_neighborhood(self.handle, C.byref(p), int(local_search), stream or None,
                                            labels.ctypes.data, C.byref(res)))
        return PbilsResult.from_c(res, labels[: self.n])

    def close(self) -> None:
        if self.handle:
            lib().ccb_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def evaluate_labelings(bits_ptr: int, n: int, words_per_row: int, edges: int, k: int, count: int, labels_ptr: int,
                       f_ptr: int, sizes_ptr: int | None = None, g_ptr: int | None = None, stream: int = 0) -> None:
    """Device recount of `count` labelings (ccb_evaluate_labelings); all pointers are device pointers."""
    check(lib().ccb_evaluate_labelings(bits_ptr, n, words_per_row, edges, k, count, labels_ptr, f_ptr, sizes_ptr,
                                       g_ptr, stream or None))


def evaluate_labelings_noalloc(bits_ptr: int, n: int, words_per_row: int, edges: int, k: int, count: int,
                               labels_ptr: int, f_ptr: int, sizes_ptr: int | None = None, g_ptr: int | None = None,
                               stream: int = 0) -> None:
    """ccb_evaluate_labelings_noalloc: the same recount for callers that cannot allocate device memory;
    its scratch is a fixed 4 MiB device array (count * k * ceil(n / 32) <= 1048576 mask words)."""
    check(lib().ccb_evaluate_labelings_noalloc(bits_ptr, n, words_per_row, edges, k, count, labels_ptr, f_ptr,
                                               sizes_ptr, g_ptr, stream or None))


def evaluate_labelings_tensor(bits_ptr: int, n: int, words_per_row: int, edges: int, k: int, count: int,
                              labels_ptr: int, f_ptr: int, sizes_ptr: int | None = None, g_ptr: int | None = None,
                              stream: int = 0) -> None:
    """ccb_evaluate_labelings_tensor: the recount with G = A*Z on the tensor cores (same outputs)."""
    check(lib().ccb_evaluate_labelings_tensor(bits_ptr, n, words_per_row, edges, k, count, labels_ptr, f_ptr,
                                              sizes_ptr, g_ptr, stream or None))


TUNING_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
TUNING_FIELDS = ("kind", "n_min", "n_max", "k_min", "k_max", "use_kind", "threads", "blocks_per_sm", "max_slots")
_tuning_loaded = False


def set_tuning(entries: list) -> None:
    """Installs a batched-engine tuning table (ccb_tuning_set): a list of dicts with TUNING_FIELDS."""
    arr = (CcbTuningEntry * max(len(entries), 1))()
    for i, e in enumerate(entries):
        arr[i] = CcbTuningEntry(*[int(e[f]) for f in TUNING_FIELDS])
    check(lib().ccb_tuning_set(arr, len(entries)))


def get_tuning() -> list:
    count = C.c_int32()
    check(lib().ccb_tuning_get(None, 0, C.byref(count)))
    arr = (CcbTuningEntry * max(count.value, 1))()
    check(lib().ccb_tuning_get(arr, count.value, C.byref(count)))
    return [{f: getattr(arr[i], f) for f in TUNING_FIELDS} for i in range(count.value)]


def load_tuning(path: str | None = None) -> bool:
    """Installs the committed table written by cuda_graph_clustering_b200.autotune (tuning.json beside this
    module) if present; returns whether one was installed.  Batch and Server call it once on first use."""
    global _tuning_loaded
    _tuning_loaded = True
    path = path or TUNING_PATH
    if not os.path.exists(path):
        return False
    with open(path) as f:
        set_tuning(json.load(f)["entries"])
    return True


def _ensure_tuning() -> None:
    if not _tuning_loaded:
        load_tuning()


BATCH_ENGINES = {"flow": 0, "lockstep": 1}


class Batch:
    """Many independent PBILS instances solved together (ccb_batch_*) by persistent per-bucket kernels fed by
    device work queues: the lock-step engine (default; one CUDA graph replay per iteration of all instances) or
    the flow engine (every instance advances on its own).  Each result equals the instance's plain solve bit
    for bit."""

    def __init__(self, engine: str = "lockstep", wait_limit_sec: float = 0.0):
        _ensure_tuning()
        h = C.c_void_p()
        check(lib().ccb_batch_create(C.byref(h)))
        self.handle = h
        self.graphs = []
        self.sizes = []
        check(lib().ccb_batch_set_engine(h, BATCH_ENGINES[engine], wait_limit_sec))

    def withhold(self, i: int) -> None:
        """Never publish instance i's work (host-side fault injection: the run ends in CCB_ERR_TIMEOUT)."""
        check(lib().ccb_batch_withhold(self.handle, i))

    def add(self, graph: DeviceGraph, params: PbilsParams) -> int:
        p = params.to_c()
        i = C.c_int32()
        check(lib().ccb_batch_add(self.handle, graph.handle, C.byref(p), C.byref(i)))
        self.graphs.append(graph)
        self.sizes.append(graph.n)
        return int(i.value)

    def run(self) -> None:
        check(lib().ccb_batch_run(self.handle))

    def result(self, i: int) -> PbilsResult:
        n = self.sizes[i]
        labels = np.zeros(max(n, 1), np.int32)
        res = CcbResult()
        check(lib().ccb_batch_result(self.handle, i, labels.ctypes.data, C.byref(res)))
        return PbilsResult.from_c(res, labels[:n])

    def describe(self) -> str:
        return lib().ccb_batch_describe(self.handle).decode()

    def close(self) -> None:
        if self.handle:
            lib().ccb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """A request loop with continuous batching (ccb_server_*): submitted requests queue FIFO, are admitted
    while their device memory fits the budget, advance one PBILS iteration per step together with every
    other admitted request, and retire when they finish.  Each result equals the request's plain solve."""

    def __init__(self, hbm_budget_bytes: int = 0, max_active: int = 0):
        _ensure_tuning()
        h = C.c_void_p()
        check(lib().ccb_server_create(hbm_budget_bytes, max_active, C.byref(h)))
        self.handle = h
        self.sizes = {}
        self._ids = (C.c_int32 * 4096)()

    def submit(self, graph: Graph, params: PbilsParams) -> int:
        p = params.to_c()
        i = C.c_int32()
        bits = np.ascontiguousarray(graph.bits, dtype=np.uint32)
        check(lib().ccb_server_submit(self.handle, bits.ctypes.data if graph.n else None, graph.n,
                                      graph.WordsPerRow(), graph.edges, C.byref(p), C.byref(i)))
        self.sizes[int(i.value)] = graph.n
        return int(i.value)

    def submit_generated(self, params: PbilsParams, n: int, density: float = 0.0, seed: int = 0,
                         planted: bool = False, parts: int = 2, p_in: float = 0.0, p_out: float = 0.0,
                         flip: float = 0.0) -> int:
        """A request whose graph is generated on the device at admission: Erdős–Rényi(n, density, seed), or
        with planted=True the planted partition(n, parts, p_in, p_out, flip, seed)."""
        p = params.to_c()
        i = C.c_int32()
        check(lib().ccb_server_submit_generated(self.handle, 1 if planted else 0, n, p_in if planted else density,
                                                p_out, flip, parts, seed, C.byref(p), C.byref(i)))
        self.sizes[int(i.value)] = n
        return int(i.value)

    def step(self) -> list:
        """Admission, one iteration of every active request, retirement; returns the ids finished."""
        count = C.c_int32()
        check(lib().ccb_server_step(self.handle, self._ids, len(self._ids), C.byref(count)))
        return [int(self._ids[j]) for j in range(min(count.value, len(self._ids)))]

    def status(self) -> tuple:
        """(queued, active, device bytes held by active requests)."""
        q, a, b = C.c_int32(), C.c_int32(), C.c_uint64()
        check(lib().ccb_server_status(self.handle, C.byref(q), C.byref(a), C.byref(b)))
        return int(q.value), int(a.value), int(b.value)

    def result(self, i: int) -> PbilsResult | None:
        """The finished request's result (released from the server), or None while it runs."""
        n = self.sizes[i]
        labels = np.zeros(max(n, 1), np.int32)
        res = CcbResult()
        done = C.c_int32()
        check(lib().ccb_server_result(self.handle, i, C.byref(done), labels.ctypes.data, C.byref(res)))
        if not done.value:
            return None
        del self.sizes[i]
        return PbilsResult.from_c(res, labels[:n])

    def cancel(self, i: int) -> bool:
        """Cancels request i (ccb_server_cancel); its result then raises CcbError with CCB_ERR_CANCELLED.
        Returns whether the request was found unfinished."""
        found = C.c_int32()
        check(lib().ccb_server_cancel(self.handle, i, C.byref(found)))
        return bool(found.value)

    def drain(self) -> dict:
        """Steps until no request is queued or active; returns {id: result} for every request finished."""
        out = {}
        while True:
            for i in self.step():
                out[i] = self.result(i)
            q, a, _ = self.status()
            if q == 0 and a == 0:
                return out

    def close(self) -> None:
        if self.handle:
            lib().ccb_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
