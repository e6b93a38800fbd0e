"""Seeded synthetic workloads (include/bingo_gen.h): R-MAT graphs, weight
distributions and update batches. These stand in for the reference's dataset
files (include/graph.cuh:22-27) and its update generators
(include/graph.cuh:58-92), which need data that is not available."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import SIGNATURES, lib

_bound = None


def bind(cdll) -> None:
    """Take the generators from another library that exports the same
    bingo_gen_* / bingo_updgen_* / bingo_edge_list_read / bingo_driver_weights
    symbols (compiled from the same gen.cpp); None returns to libbingo.so.
    A CPU-only caller uses this to build workloads without loading the engine."""
    global _bound
    if cdll is not None:
        for name, (res, args) in SIGNATURES.items():
            if name.startswith(("bingo_gen_", "bingo_updgen_", "bingo_edge_list_", "bingo_driver_weights")):
                f = getattr(cdll, name)
                f.restype = res
                f.argtypes = args
    _bound = cdll


def _lib():
    return _bound if _bound is not None else lib()


W_UNIFORM, W_LOGUNIFORM, W_ZIPF = 0, 1, 2
DRIVER_AUTO, DRIVER_DEGREE, DRIVER_DEGREE_POW03 = 0, 1, 2
_READ_ERRORS = {-1: "cannot open or read", -2: "malformed token", -3: "arrays too small", -4: "id above 2^32 - 2"}


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1):
    """R-MAT edges (src, dst) as uint32, sorted by (src, dst), no self-loops or duplicates."""
    cap = edge_factor << scale
    src = np.empty(cap, np.uint32)
    dst = np.empty(cap, np.uint32)
    m = _lib().bingo_gen_rmat(scale, edge_factor, a, b, c, seed, _p(src), _p(dst))
    return src[:m].copy(), dst[:m].copy()


def weights(m: int, dist: int = W_UNIFORM, lo: float = 1, hi: float = 1024, s: float = 1.2, seed: int = 2):
    w = np.empty(m, np.uint32)
    _lib().bingo_gen_weights(m, dist, lo, hi, s, seed, _p(w))
    return w


class UpdateGen:
    """Absent-pair inserts and uniform live-edge deletes, tracking slots the
    way the engine assigns them (append order per vertex)."""

    def __init__(self, n: int, src: np.ndarray, dst: np.ndarray, seed: int = 3):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        self._L = _lib()
        self._g = self._L.bingo_updgen_create(n, _p(src), _p(dst), len(src), seed)

    def inserts(self, k: int, dist: int = W_UNIFORM, lo: float = 1, hi: float = 1024, s: float = 1.2):
        src = np.empty(k, np.uint32)
        dst = np.empty(k, np.uint32)
        w = np.empty(k, np.uint32)
        self._L.bingo_updgen_inserts(self._g, k, dist, lo, hi, s, _p(src), _p(dst), _p(w))
        return src, dst, w

    def deletes(self, k: int):
        u = np.empty(k, np.uint32)
        slot = np.empty(k, np.uint32)
        made = self._L.bingo_updgen_deletes(self._g, k, _p(u), _p(slot))
        return u[:made].copy(), slot[:made].copy()

    @property
    def live(self) -> int:
        return self._L.bingo_updgen_live(self._g)

    def __del__(self):
        if getattr(self, "_g", None):
            self._L.bingo_updgen_destroy(self._g)
            self._g = None


def read_edge_list(path: str):
    """An edge-list file as the reference's loadGraph() reads it ("u v" pairs,
    include/graph.cuh:22-27; '#'/'%' comment lines skipped). Returns
    (src, dst, n) with ids as in the file and n = largest id + 1."""
    L = _lib()
    m, n = ctypes.c_uint64(), ctypes.c_uint32()
    bp = os.fsencode(path)
    rc = L.bingo_edge_list_read(bp, None, None, 0, ctypes.byref(m), ctypes.byref(n))
    if rc:
        raise ValueError(f"{path}: {_READ_ERRORS.get(rc, rc)}" + (f" at byte {m.value}" if rc == -2 else ""))
    src = np.empty(m.value, np.uint32)
    dst = np.empty(m.value, np.uint32)
    rc = L.bingo_edge_list_read(bp, _p(src), _p(dst), len(src), ctypes.byref(m), ctypes.byref(n))
    if rc:
        raise ValueError(f"{path}: {_READ_ERRORS.get(rc, rc)}")
    return src, dst, int(n.value)


def driver_weights(src, dst, n: int, kind: int = DRIVER_AUTO):
    """The reference driver's load weights: trunc(bias(outdeg(v))) + 1 with
    bias(d) = d, or d^0.3 for n > 1e7 (include/graph.cuh:43-51, include/api.h:29-30)."""
    s, d = np.ascontiguousarray(src, np.uint32), np.ascontiguousarray(dst, np.uint32)
    w = np.empty(len(s), np.uint32)
    if _lib().bingo_driver_weights(kind, _p(s), _p(d), len(s), n, _p(w)):
        raise ValueError("unknown weight kind or an id >= n")
    return w

