"""ctypes wrapper over oracle/liboracle.so (the CPU oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker; the product never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp = c_void_p
        sig = {
            "orc_philox": (None, [vp, vp, vp]),
            "orc_alias_build": (c_int, [vp, vp, vp, vp, vp]),
            "orc_walk_thresholds": (None, [c_double, c_double, c_double, vp, vp]),
            "orc_new": (vp, [c_uint32]),
            "orc_free": (None, [vp]),
            "orc_load": (None, [vp, vp, vp, vp, c_uint64]),
            "orc_insert": (None, [vp, vp, vp, vp, c_uint64, vp]),
            "orc_delete": (c_uint64, [vp, vp, vp, c_uint64]),
            "orc_delete_pairs": (c_uint64, [vp, vp, vp, c_uint64, vp]),
            "orc_walk": (None, [vp, c_int, c_uint32, vp, c_uint64, c_uint64, c_uint32, c_double, c_double,
                                c_double, c_uint32, vp]),
            "orc_walk_interleaved": (None, [vp, c_int, c_uint32, vp, c_uint64, c_uint64, c_uint32, c_double, vp]),
            "orc_has_edge": (c_int, [vp, c_uint32, c_uint32]),
            "orc_dump_sizes": (None, [vp, vp]),
            "orc_dump": (None, [vp] * 14),
            "orl_new": (vp, [c_uint32, c_float]),
            "orl_free": (None, [vp]),
            "orl_load": (None, [vp, vp, vp, vp, c_uint64]),
            "orl_insert": (None, [vp, vp, vp, vp, c_uint64]),
            "orl_delete": (None, [vp, vp, vp, c_uint64]),
            "orl_dump_sizes": (None, [vp, vp]),
            "orl_dump": (None, [vp] * 16),
            "orl_implied_probs": (None, [vp, c_uint32, vp]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _L = L
    return _L


def gen_lib():
    """This library as a source of the seeded workload generators (the same
    gen.cpp the engine library compiles, linked into liboracle.so), for
    callers that must not load the engine (bingo_b200.gen.bind)."""
    return lib()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def philox(ctr, key):
    """Philox4x32-10 of one 4-word counter under a 2-word key."""
    c = _u32(ctr)
    k = _u32(key)
    o = np.zeros(4, np.uint32)
    lib().orc_philox(_p(c), _p(k), _p(o))
    return o


def alias_build(mass32):
    mass = np.ascontiguousarray(mass32, dtype=np.uint64)
    thr = np.zeros(32, np.uint64)
    T = np.zeros(32, np.uint64)
    own = np.zeros(32, np.uint8)
    al = np.zeros(32, np.uint8)
    m = lib().orc_alias_build(_p(mass), _p(thr), _p(T), _p(own), _p(al))
    return m, thr[:m], T[:m], own[:m], al[:m]


def walk_thresholds(p, q, stop):
    o = np.zeros(4, np.uint64)
    ex = np.zeros(1, np.float64)
    lib().orc_walk_thresholds(p, q, stop, _p(o), _p(ex))
    return o, float(ex[0])


class ExactGraph:
    """The integer semantics the CUDA path implements."""

    def __init__(self, n: int):
        self.n = n
        self._g = lib().orc_new(n)

    def __del__(self):
        if getattr(self, "_g", None):
            lib().orc_free(self._g)
            self._g = None

    def load(self, src, dst, w):
        s, d, ww = _u32(src), _u32(dst), _u32(w)
        lib().orc_load(self._g, _p(s), _p(d), _p(ww), len(s))

    def insert(self, src, dst, w):
        s, d, ww = _u32(src), _u32(dst), _u32(w)
        out = np.zeros(len(s), np.uint32)
        lib().orc_insert(self._g, _p(s), _p(d), _p(ww), len(s), _p(out))
        return out

    def delete(self, u, slot):
        uu, ss = _u32(u), _u32(slot)
        return lib().orc_delete(self._g, _p(uu), _p(ss), len(uu))

    def delete_pairs(self, u, v):
        """Returns (rejected count, translated slot per pair)."""
        uu, vv = _u32(u), _u32(v)
        out = np.zeros(len(uu), np.uint32)
        bad = lib().orc_delete_pairs(self._g, _p(uu), _p(vv), len(uu), _p(out))
        return bad, out

    def walk(self, app, length, starts, seed=0, job_id=0, p=0.5, q=2.0, stop=0.0125, flags=0):
        st = _u32(starts)
        out = np.zeros(len(st) if app == 3 else len(st) * length, np.int32)
        lib().orc_walk(self._g, app, length, _p(st), len(st), seed, job_id, p, q, stop, flags, _p(out))
        return out if app == 3 else out.reshape(len(st), length)

    def walk_interleaved(self, app, length, starts, seed=0, job_id=0, stop=0.0125):
        """walk() for DeepWalk and PPR (no tail flag) with several walks per
        thread in flight: the same rows, faster; the timed CPU baseline."""
        if app not in (0, 2):
            raise ValueError("walk_interleaved runs DeepWalk and PPR only")
        st = _u32(starts)
        out = np.zeros(len(st) * length, np.int32)
        lib().orc_walk_interleaved(self._g, app, length, _p(st), len(st), seed, job_id, stop, _p(out))
        return out.reshape(len(st), length)

    def has_edge(self, u, v):
        return bool(lib().orc_has_edge(self._g, u, v))

    def dump(self):
        sz = np.zeros(3, np.uint64)
        lib().orc_dump_sizes(self._g, _p(sz))
        ns, nm, na = (int(x) for x in sz)
        n = self.n
        d = dict(
            ecnt=np.zeros(n, np.uint32), live=np.zeros(n, np.uint32), ev=np.zeros(ns, np.uint32),
            ew=np.zeros(ns, np.uint32), gcnt=np.zeros(n * 32, np.uint32), mslot=np.zeros(nm, np.uint32),
            mv=np.zeros(nm, np.uint32), mbp=np.zeros(nm, np.uint32), am=np.zeros(n, np.uint32),
            athr=np.zeros(na, np.uint64), aT=np.zeros(na, np.uint64), aown=np.zeros(na, np.uint8),
            aalias=np.zeros(na, np.uint8))
        order = ["ecnt", "live", "ev", "ew", "gcnt", "mslot", "mv", "mbp", "am", "athr", "aT", "aown", "aalias"]
        lib().orc_dump(self._g, *[_p(d[k]) for k in order])
        return d


REF_DUMP_FIELDS = ["logt", "bits", "sz", "ecnt", "asz", "ev", "ew", "grouptp", "num", "gsz", "members", "midx",
                   "ap", "aa", "ab"]
REF_DUMP_DTYPES = dict(logt=np.int32, bits=np.int32, sz=np.int32, ecnt=np.uint32, asz=np.uint32, ev=np.uint32,
                       ew=np.float32, grouptp=np.int8, num=np.float32, gsz=np.uint32, members=np.uint32,
                       midx=np.int32, ap=np.float32, aa=np.int8, ab=np.int8)


class RefGraph:
    """The reference's NodeData state machine restated on the CPU."""

    def __init__(self, n: int, rate: float = 0.4):
        self.n = n
        self._g = lib().orl_new(n, rate)

    def __del__(self):
        if getattr(self, "_g", None):
            lib().orl_free(self._g)
            self._g = None

    def load(self, src, dst, w):
        s, d, ww = _u32(src), _u32(dst), _u32(w)
        lib().orl_load(self._g, _p(s), _p(d), _p(ww), len(s))

    def insert(self, src, dst, w):
        s, d, ww = _u32(src), _u32(dst), _u32(w)
        lib().orl_insert(self._g, _p(s), _p(d), _p(ww), len(s))

    def delete(self, u, slot):
        uu, ss = _u32(u), _u32(slot)
        lib().orl_delete(self._g, _p(uu), _p(ss), len(uu))

    def implied_probs(self, u):
        o = np.zeros(32, np.float64)
        lib().orl_implied_probs(self._g, u, _p(o))
        return o

    def dump(self):
        sz = np.zeros(5, np.uint64)
        lib().orl_dump_sizes(self._g, _p(sz))
        ns, nl, nb, nm, na = (int(x) for x in sz)
        n = self.n
        sizes = dict(logt=n, bits=n, sz=n, ecnt=n, asz=n, ev=ns, ew=ns, grouptp=nl, num=nl, gsz=nb, members=nm,
                     midx=nm, ap=na, aa=na, ab=na)
        d = {k: np.zeros(sizes[k], REF_DUMP_DTYPES[k]) for k in REF_DUMP_FIELDS}
        lib().orl_dump(self._g, *[_p(d[k]) for k in REF_DUMP_FIELDS])
        return d


def read_ref_dumps(path):
    """Parse the dumps the reference harness (oracle/ref_harness.cu) writes."""
    out = []
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0
    while pos < len(buf):
        assert buf[pos:pos + 4] == b"DUMP", "bad dump block"
        pos += 4
        n = int(np.frombuffer(buf, np.uint32, 1, pos)[0])
        pos += 4
        d = {"n": n}
        for k in REF_DUMP_FIELDS:
            cnt = int(np.frombuffer(buf, np.uint64, 1, pos)[0])
            pos += 8
            dt = np.dtype(REF_DUMP_DTYPES[k])
            d[k] = np.frombuffer(buf, dt, cnt, pos).copy()
            pos += cnt * dt.itemsize
        out.append(d)
    return out
