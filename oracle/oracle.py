"""ctypes access to the CPU checkers (test infrastructure only).

``Oracle`` wraps ``oracle/liboracle.so``, the plain-C restatement of the reference CPU solver
(``src/cc_pbils_cpu.cpp``, ``include/cc_math.hpp``, ``src/cc_graph.cpp``).  ``Reference`` wraps
``oracle/_ref/libccref.so``, the reference's own CPU sources compiled by ``oracle/Makefile``.
Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libccref.so")
REF_CPU_BIN = os.path.join(HERE, "_ref", "cc_cpu")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


class Params(C.Structure):
    """Mirror of the PBILS knobs of cc::PbilsParams (include/cc_pbils.hpp:26-49)."""

    _fields_ = [("k", C.c_int32), ("population", C.c_int32), ("tournament", C.c_int32),
                ("iterations", C.c_int32), ("early_stop", C.c_int32), ("perturbation", C.c_double),
                ("gww", C.c_double), ("seed", C.c_uint64)]


class Result(C.Structure):
    _fields_ = [("objective", C.c_int64), ("iterations_done", C.c_int32), ("clusters_used", C.c_int32),
                ("local_searches", C.c_int64), ("accepted_moves", C.c_int64)]


@dataclass
class Solution:
    objective: int
    labels: np.ndarray
    iterations_done: int
    clusters_used: int
    local_searches: int
    accepted_moves: int
    trace: np.ndarray | None = None


def words_per_row(n: int) -> int:
    return 1 if n == 0 else (n + 31) // 32


def make_params(k=2, population=128, tournament=5, iterations=100, early_stop=6, perturbation=0.4, gww=0.1,
                seed=1) -> Params:
    """Defaults of cc::PbilsParams (include/cc_pbils.hpp:32-43)."""
    return Params(k, population, tournament, iterations, early_stop, perturbation, gww, seed)


def ensure_built() -> None:
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)


class Oracle:
    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            ensure_built()
        lib = C.CDLL(path)
        self.lib = lib
        lib.orc_stream_seed.restype = C.c_uint64
        lib.orc_stream_seed.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        lib.orc_initial_label.restype = C.c_int
        lib.orc_initial_label.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
        lib.orc_tournament.restype = C.c_int
        lib.orc_tournament.argtypes = [C.c_uint64, C.c_int, C.c_int, _i64p, C.c_int, C.c_int]
        lib.orc_perturbed_label.restype = C.c_int
        lib.orc_perturbed_label.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_float]
        lib.orc_erdos_renyi.restype = C.c_uint64
        lib.orc_erdos_renyi.argtypes = [C.c_uint32, C.c_double, C.c_uint64, _u32p]
        lib.orc_planted.restype = C.c_uint64
        lib.orc_planted.argtypes = [C.c_uint32, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                    _u32p, _i32p]
        lib.orc_objective_direct.restype = C.c_int64
        lib.orc_objective_direct.argtypes = [_u32p, C.c_uint32, C.c_uint32, _i32p]
        lib.orc_objective_bitwise.restype = C.c_int64
        lib.orc_objective_bitwise.argtypes = [_u32p, C.c_uint32, C.c_uint32, _i32p]
        lib.orc_rebuild.restype = C.c_int64
        lib.orc_rebuild.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int, _i32p, _i32p, _i32p]
        lib.orc_local_search.restype = C.c_int64
        lib.orc_local_search.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int, _i32p, _i64p]
        lib.orc_winner_copies.restype = C.c_int
        lib.orc_winner_copies.argtypes = [C.c_double, C.c_int]
        lib.orc_rank_slots.restype = None
        lib.orc_rank_slots.argtypes = [_i64p, C.c_int, _i32p]
        lib.orc_pbils.restype = C.c_int
        lib.orc_pbils.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(Params), C.c_int, _i32p,
                                  C.POINTER(Result), C.c_void_p]
        lib.orc_neighborhood.restype = C.c_int
        lib.orc_neighborhood.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int, C.c_int, _i32p,
                                         C.POINTER(Result)]

    # --- graphs -----------------------------------------------------------------------------
    def erdos_renyi(self, n: int, density: float, seed: int):
        bits = np.zeros(n * words_per_row(n), np.uint32)
        edges = self.lib.orc_erdos_renyi(n, density, seed, bits)
        return bits.reshape(n, words_per_row(n)), int(edges)

    def planted(self, n: int, parts: int, shuffle_split: bool, p_in: float, p_out: float, flip: float, seed: int):
        bits = np.zeros(max(1, n * words_per_row(n)), np.uint32)
        community = np.zeros(max(1, n), np.int32)
        edges = self.lib.orc_planted(n, parts, int(shuffle_split), p_in, p_out, flip, seed, bits, community)
        return bits[: n * words_per_row(n)].reshape(n, words_per_row(n)), int(edges), community[:n]

    # --- objective / state ------------------------------------------------------------------
    @staticmethod
    def _flat(bits):
        return np.ascontiguousarray(bits, dtype=np.uint32).reshape(-1)

    def objective_direct(self, bits, labels):
        n = bits.shape[0]
        return int(self.lib.orc_objective_direct(self._flat(bits), n, bits.shape[1],
                                                 np.ascontiguousarray(labels, np.int32)))

    def objective_bitwise(self, bits, labels):
        n = bits.shape[0]
        return int(self.lib.orc_objective_bitwise(self._flat(bits), n, bits.shape[1],
                                                  np.ascontiguousarray(labels, np.int32)))

    def rebuild(self, bits, edges, k, labels):
        n = bits.shape[0]
        g = np.zeros(max(1, k * n), np.int32)
        sizes = np.zeros(k, np.int32)
        f = self.lib.orc_rebuild(self._flat(bits), n, bits.shape[1], edges, k,
                                 np.ascontiguousarray(labels, np.int32), g, sizes)
        return int(f), g[: k * n].reshape(k, n), sizes

    def local_search(self, bits, edges, k, labels):
        n = bits.shape[0]
        lab = np.array(labels, np.int32, copy=True)
        moves = np.zeros(1, np.int64)
        f = self.lib.orc_local_search(self._flat(bits), n, bits.shape[1], edges, k, lab, moves)
        return int(f), lab, int(moves[0])

    def rank_slots(self, f):
        f = np.ascontiguousarray(f, np.int64)
        order = np.zeros(len(f), np.int32)
        self.lib.orc_rank_slots(f, len(f), order)
        return order

    # --- solvers ----------------------------------------------------------------------------
    def pbils(self, bits, edges, params: Params, threads: int = 0, trace: bool = False) -> Solution:
        n = bits.shape[0]
        labels = np.zeros(max(1, n), np.int32)
        res = Result()
        tr = np.zeros(max(1, params.iterations), np.int64) if trace else None
        threads = threads if threads > 0 else (os.cpu_count() or 1)
        rc = self.lib.orc_pbils(self._flat(bits), n, bits.shape[1], edges, C.byref(params), threads, labels,
                                C.byref(res), tr.ctypes.data if trace else None)
        if rc != 0:
            raise RuntimeError("invalid PBILS parameters")
        return Solution(res.objective, labels[:n], res.iterations_done, res.clusters_used, res.local_searches,
                        res.accepted_moves, tr[: res.iterations_done] if trace else None)

    def neighborhood(self, bits, edges, local_search: bool, threads: int = 0) -> Solution:
        n = bits.shape[0]
        labels = np.zeros(max(1, n), np.int32)
        res = Result()
        threads = threads if threads > 0 else (os.cpu_count() or 1)
        rc = self.lib.orc_neighborhood(self._flat(bits), n, bits.shape[1], edges, int(local_search), threads, labels,
                                       C.byref(res))
        if rc != 0:
            raise RuntimeError("Neighborhood requires n >= 1")
        return Solution(res.objective, labels[:n], 0, res.clusters_used, res.local_searches, res.accepted_moves)


class Reference:
    """The reference's own CPU solver, compiled by oracle/Makefile into oracle/_ref/libccref.so."""

    def __init__(self, path: str = REF_LIB_PATH):
        lib = C.CDLL(path)
        self.lib = lib
        lib.ref_erdos_renyi.restype = C.c_uint64
        lib.ref_erdos_renyi.argtypes = [C.c_uint32, C.c_double, C.c_uint64, _u32p]
        lib.ref_pbils.restype = C.c_int
        lib.ref_pbils.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.POINTER(Params), C.c_int, _i32p, C.POINTER(Result)]
        lib.ref_rebuild.restype = C.c_int64
        lib.ref_rebuild.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_int, _i32p, _i32p, _i32p]
        lib.ref_local_search.restype = C.c_int64
        lib.ref_local_search.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_int, _i32p, _i64p]
        lib.ref_neighborhood.restype = C.c_int
        lib.ref_neighborhood.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_int, _i32p, C.POINTER(Result)]
        lib.ref_neighborhood_range.restype = C.c_int64
        lib.ref_neighborhood_range.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32, _i64p]
        lib.ref_load_tags.restype = C.c_int64
        lib.ref_load_tags.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_uint32, C.c_uint64, C.c_uint32, _u32p,
                                      C.POINTER(C.c_uint64)]
        lib.ref_objective_direct.restype = C.c_int64
        lib.ref_objective_direct.argtypes = [_u32p, C.c_uint32, C.c_uint32, _i32p]
        lib.ref_objective_bitwise.restype = C.c_int64
        lib.ref_objective_bitwise.argtypes = [_u32p, C.c_uint32, C.c_uint32, _i32p]
        lib.ref_rank_slots.restype = None
        lib.ref_rank_slots.argtypes = [_i64p, C.c_int, _i32p]
        lib.ref_tournament.restype = C.c_int
        lib.ref_tournament.argtypes = [C.c_uint64, C.c_int, C.c_int, _i64p, C.c_int, C.c_int]
        lib.ref_perturbed_label.restype = C.c_int
        lib.ref_perturbed_label.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_float]
        lib.ref_initial_label.restype = C.c_int
        lib.ref_initial_label.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
        lib.ref_stream_seed.restype = C.c_uint64
        lib.ref_stream_seed.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_LIB_PATH)

    def erdos_renyi(self, n, density, seed):
        bits = np.zeros(n * words_per_row(n), np.uint32)
        edges = self.lib.ref_erdos_renyi(n, density, seed, bits)
        return bits.reshape(n, words_per_row(n)), int(edges)

    def pbils(self, bits, params: Params, threads: int = 0) -> Solution:
        n = bits.shape[0]
        labels = np.zeros(max(1, n), np.int32)
        res = Result()
        threads = threads if threads > 0 else (os.cpu_count() or 1)
        rc = self.lib.ref_pbils(np.ascontiguousarray(bits, np.uint32).reshape(-1), n, bits.shape[1],
                                C.byref(params), threads, labels, C.byref(res))
        if rc != 0:
            raise RuntimeError("reference rejected the parameters")
        return Solution(res.objective, labels[:n], res.iterations_done, res.clusters_used, res.local_searches,
                        res.accepted_moves)

    def neighborhood(self, bits, local_search: bool) -> Solution:
        n = bits.shape[0]
        labels = np.zeros(max(1, n), np.int32)
        res = Result()
        self.lib.ref_neighborhood(np.ascontiguousarray(bits, np.uint32).reshape(-1), n, bits.shape[1],
                                  int(local_search), labels, C.byref(res))
        return Solution(res.objective, labels[:n], 0, res.clusters_used, res.local_searches, res.accepted_moves)

    def neighborhood_range(self, bits, local_search: bool, first: int, count: int):
        """The brute force over start vertices [first, first + count) only: (best f, accepted moves)."""
        best = np.zeros(1, np.int64)
        moves = self.lib.ref_neighborhood_range(np.ascontiguousarray(bits, np.uint32).reshape(-1), bits.shape[0],
                                                bits.shape[1], int(local_search), first, count, best)
        return int(best[0]), int(moves)

    def load_tags(self, path: str, similarity: str, threshold: float, n: int, seed: int, capacity: int):
        """The reference's own Graph::LoadTags: (bits [n][words_per_row], edges)."""
        bits = np.zeros(max(1, capacity * words_per_row(capacity)), np.uint32)
        edges = C.c_uint64()
        size = self.lib.ref_load_tags(path.encode(), similarity.encode(), threshold, n, seed, capacity, bits,
                                      C.byref(edges))
        if size < 0:
            raise RuntimeError("reference LoadTags failed")
        size = int(size)
        return bits[: size * words_per_row(size)].reshape(size, words_per_row(size)), int(edges.value)

    def rebuild(self, bits, k, labels):
        n = bits.shape[0]
        g = np.zeros(max(1, k * n), np.int32)
        sizes = np.zeros(k, np.int32)
        f = self.lib.ref_rebuild(np.ascontiguousarray(bits, np.uint32).reshape(-1), n, bits.shape[1], k,
                                 np.ascontiguousarray(labels, np.int32), g, sizes)
        return int(f), g[: k * n].reshape(k, n), sizes

    def local_search(self, bits, k, labels):
        n = bits.shape[0]
        lab = np.array(labels, np.int32, copy=True)
        moves = np.zeros(1, np.int64)
        f = self.lib.ref_local_search(np.ascontiguousarray(bits, np.uint32).reshape(-1), n, bits.shape[1], k, lab,
                                      moves)
        return int(f), lab, int(moves[0])
