"""Host-side interface of the B200 walk engine.

`Graph` mirrors the reference's operator surface (include/operation.cuh:
``build`` :33, ``insert`` :144, ``deleteE`` :215 and the walk kernels
:252-430 launched by ``randomWalk``, include/graph.cuh:93) over the C ABI in
include/bingo.h. Arrays may be numpy arrays (host) or CUDA tensors (device);
ids are 0-based. Errors raise `BingoError` carrying the C status.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from ._lib import (CHECK_KINDS, TUNING_FIELDS, BingoCheckReport, BingoConfig, BingoError, BingoOp,
                   BingoServeConfig, BingoServeMetrics, BingoServeStatus, BingoStats, BingoTuneReport, BingoTuneRequest, BingoTuning, BingoWalkJob, lib)

DEEPWALK, NODE2VEC, PPR, SAMPLING = 0, 1, 2, 3
APPS = {"deepwalk": DEEPWALK, "node2vec": NODE2VEC, "ppr": PPR, "sampling": SAMPLING}
WALK_PPR_TAIL = 1
BATCHED, PLAIN = 0, 1
OP_WALK, OP_INSERT, OP_DELETE, OP_DELETE_PAIRS = 0, 1, 2, 3
RUN_GRAPH = 1


def _read_json(path) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _is_float(a) -> bool:
    if hasattr(a, "dtype") and hasattr(a, "data_ptr"):
        return a.dtype.is_floating_point
    return np.asarray(a).dtype.kind == "f"


def _f32(a):
    """Pointer + keep-alive for a float32 array (numpy host array or CUDA tensor)."""
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous() or a.element_size() != 4:
            raise ValueError("expected a contiguous float32 tensor")
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.ascontiguousarray(a, dtype=np.float32)
    return ctypes.c_void_p(arr.ctypes.data), arr


def fixed16(w) -> np.ndarray:
    """Float weights -> the float-weight mode's 16.16 fixed point (bingo_weights_to_fixed16); invalid -> 0."""
    arr = np.ascontiguousarray(w, dtype=np.float32)
    out = np.empty(len(arr), np.uint32)
    lib().bingo_weights_to_fixed16(ctypes.c_void_p(arr.ctypes.data), len(arr), ctypes.c_void_p(out.ctypes.data))
    return out


def _u32(a):
    """Pointer + keep-alive for a uint32 array (numpy host array or CUDA tensor)."""
    if a is None:
        return None, None
    if hasattr(a, "data_ptr"):  # torch tensor
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        if a.element_size() != 4:
            raise ValueError("expected a 32-bit tensor")
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.ascontiguousarray(a, dtype=np.uint32)
    return ctypes.c_void_p(arr.ctypes.data), arr


def _out(a, dtype):
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr()), a
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous):
        raise ValueError(f"output must be a contiguous numpy {np.dtype(dtype)} array or a tensor")
    return ctypes.c_void_p(a.ctypes.data), a


@dataclass
class WalkJob:
    """One walk job (bingo_walk_job). starts=None walks [first, first+n_starts)."""
    app: int = DEEPWALK
    length: int = 80
    starts: Optional[object] = None
    n_starts: int = 0
    first: int = 0
    job_id: int = 0
    seed: int = 0
    flags: int = 0
    p: float = 0.5
    q: float = 2.0
    stop_prob: float = 0.0125
    out: Optional[object] = None


class Graph:
    """A dynamic weighted graph resident on one GPU."""

    def __init__(self, device: int = 0, node2vec: bool = True, synchronous: bool = True,
                 arena_factor: float = 2.0, arena_bytes: int = 0, float_weights: bool = False):
        L = lib()
        cfg = BingoConfig()
        L.bingo_config_init(ctypes.byref(cfg))
        cfg.device = device
        cfg.weight_mode = 1 if float_weights else 0
        self.float_weights = float_weights
        self.device = device
        cfg.node2vec = 1 if node2vec else 0
        cfg.synchronous = 1 if synchronous else 0
        cfg.arena_factor = arena_factor
        cfg.arena_bytes = arena_bytes
        h = ctypes.c_void_p()
        st = L.bingo_create(ctypes.byref(cfg), ctypes.byref(h))
        if st:
            raise BingoError(st, (L.bingo_last_error(None) or b"").decode())
        self._h = h
        self._L = L
        self.n = 0

    # ------------------------------------------------------------------ util
    def _check(self, st: int):
        if st:
            raise BingoError(st, (self._L.bingo_last_error(self._h) or b"").decode())

    def close(self):
        """Destroy the handle (bingo_destroy): frees the graph arenas, staging
        buffers and streams. Idempotent."""
        if getattr(self, "_h", None):
            self._L.bingo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------------ ops
    def load_edges(self, src, dst, w, n: int):
        """Load a graph (reference build(), include/operation.cuh:33)."""
        ps, ks = _u32(src)
        pd, kd = _u32(dst)
        m = len(src) if not hasattr(src, "numel") else src.numel()
        if _is_float(w):  # float weights (handle created with float_weights=True)
            pw, kw = _f32(w)
            self._check(self._L.bingo_load_edges_f32(self._h, ps, pd, pw, m, n))
        else:
            pw, kw = _u32(w)
            self._check(self._L.bingo_load_edges(self._h, ps, pd, pw, m, n))
        self.n = n

    def insert_batch(self, src, dst, w, out_slots=None, return_slots: bool = True):
        """Append a batch of edges (reference insert(), include/operation.cuh:144).
        Returns the slot id of every edge (numpy) unless out_slots is given."""
        k = len(src) if not hasattr(src, "numel") else src.numel()
        ps, ks = _u32(src)
        pd, kd = _u32(dst)
        if out_slots is None and return_slots:
            out_slots = np.empty(k, dtype=np.uint32)
        po, ko = _out(out_slots, np.uint32) if out_slots is not None else (None, None)
        if _is_float(w):
            pw, kw = _f32(w)
            self._check(self._L.bingo_insert_batch_f32(self._h, ps, pd, pw, k, po))
        else:
            pw, kw = _u32(w)
            self._check(self._L.bingo_insert_batch(self._h, ps, pd, pw, k, po))
        return out_slots

    def delete_batch(self, u, slot):
        """Delete (vertex, slot) pairs (reference deleteE(), include/operation.cuh:215)."""
        k = len(u) if not hasattr(u, "numel") else u.numel()
        pu, ku = _u32(u)
        psl, ksl = _u32(slot)
        self._check(self._L.bingo_delete_batch(self._h, pu, psl, k))

    def delete_pairs(self, u, v):
        """Delete edges by (u, v): the r-th repeat of a pair takes the r-th lowest live slot (bingo_delete_pairs)."""
        k = len(u) if not hasattr(u, "numel") else u.numel()
        pu, ku = _u32(u)
        pv, kv = _u32(v)
        self._check(self._L.bingo_delete_pairs(self._h, pu, pv, k))

    @staticmethod
    def _job_array(jobs: Sequence[WalkJob], keep: list):
        arr = (BingoWalkJob * len(jobs))()
        for i, j in enumerate(jobs):
            ps, ks = _u32(j.starts) if j.starts is not None else (None, None)
            po, ko = _out(j.out, np.int32)
            keep += [ks, ko]
            arr[i].app = j.app
            arr[i].length = j.length
            arr[i].starts = ps
            arr[i].n_starts = j.n_starts
            arr[i].first = j.first
            arr[i].job_id = j.job_id
            arr[i].seed = j.seed
            arr[i].flags = j.flags
            arr[i].p = j.p
            arr[i].q = j.q
            arr[i].stop_prob = j.stop_prob
            arr[i].out = po
        return arr

    def walk_jobs(self, jobs: Sequence[WalkJob], mode: int = BATCHED):
        """Run a list of walk jobs; each job's out must be preallocated."""
        keep = []
        arr = self._job_array(jobs, keep)
        self._check(self._L.bingo_walk(self._h, arr, len(jobs), mode))

    def run(self, ops: Sequence[tuple], graph: bool = True):
        """Run a program: a list of ("walk", [WalkJob...]), ("insert", src, dst,
        w[, out_slots]), ("delete", u, slot) and ("delete_pairs", u, v) with device tensors, in order
        and without host synchronisation (bingo_run). graph=True captures it
        into a CUDA graph replayed while its shape is unchanged."""
        arr = (BingoOp * len(ops))()
        keep = []
        for i, op in enumerate(ops):
            kind = op[0]
            if kind == "walk":
                jobs = self._job_array(op[1], keep)
                keep.append(jobs)
                arr[i].kind, arr[i].n_jobs = OP_WALK, len(op[1])
                arr[i].jobs = ctypes.cast(jobs, ctypes.POINTER(BingoWalkJob))
            elif kind in ("insert", "delete", "delete_pairs"):
                cols = [_u32(x) for x in op[1:4 if kind == "insert" else 3]]
                keep += [c[1] for c in cols]
                arr[i].kind = {"insert": OP_INSERT, "delete": OP_DELETE, "delete_pairs": OP_DELETE_PAIRS}[kind]
                arr[i].a, arr[i].b = cols[0][0], cols[1][0]
                if kind == "insert":
                    arr[i].c = cols[2][0]
                    if len(op) > 4 and op[4] is not None:
                        po, ko = _out(op[4], np.uint32)
                        keep.append(ko)
                        arr[i].out_slots = po
                arr[i].k = op[1].numel() if hasattr(op[1], "numel") else len(op[1])
            else:
                raise ValueError(f"unknown op {kind!r}")
        self._check(self._L.bingo_run(self._h, arr, len(ops), RUN_GRAPH if graph else 0))

    def walk(self, app: int = DEEPWALK, length: int = 80, starts=None, n_starts: Optional[int] = None,
             first: int = 0, seed: int = 0, job_id: int = 0, p: float = 0.5, q: float = 2.0,
             stop_prob: float = 0.0125, flags: int = 0, mode: int = PLAIN, out=None):
        """One walk job; returns [n_starts][length] int32 (sampling: [n_starts])."""
        if starts is not None:
            n_starts = len(starts) if not hasattr(starts, "numel") else starts.numel()
        if n_starts is None:
            n_starts = self.n - first
        if out is None:
            out = np.empty((n_starts,) if app == SAMPLING else (n_starts, length), dtype=np.int32)
        self.walk_jobs([WalkJob(app=app, length=length, starts=starts, n_starts=n_starts, first=first,
                                job_id=job_id, seed=seed, flags=flags, p=p, q=q, stop_prob=stop_prob,
                                out=out)], mode=mode)
        return out

    # ------------------------------------------------------------ serving
    def serve_start(self, output_budget_bytes: int = 1 << 30, max_jobs: int = 4096,
                    max_update_batch: int = 1 << 20, idle_timeout_us: int = 2000):
        """Start the continuous-batching walk server (bingo_serve_start)."""
        cfg = BingoServeConfig(output_budget_bytes, max_jobs, max_update_batch, idle_timeout_us, 0)
        self._check(self._L.bingo_serve_start(self._h, ctypes.byref(cfg)))
        self._serve_keep = {}

    def submit_walk(self, app: int = DEEPWALK, length: int = 80, starts=None, n_starts: Optional[int] = None,
                    first: int = 0, seed: int = 0, job_id: int = 0, p: float = 0.5, q: float = 2.0,
                    stop_prob: float = 0.0125, flags: int = 0, out=None):
        """Submit one walk query; returns (ticket, out). out is filled when the ticket is done."""
        if starts is not None:
            n_starts = len(starts) if not hasattr(starts, "numel") else starts.numel()
        if out is None:
            out = np.empty((n_starts,) if app == SAMPLING else (n_starts, length), dtype=np.int32)
        keep = []
        job = self._job_array([WalkJob(app=app, length=length, starts=starts, n_starts=n_starts, first=first,
                                       job_id=job_id, seed=seed, flags=flags, p=p, q=q, stop_prob=stop_prob,
                                       out=out)], keep)
        t = ctypes.c_uint64()
        self._check(self._L.bingo_serve_submit_walk(self._h, job, ctypes.byref(t)))
        self._serve_keep[t.value] = out
        return t.value, out

    def submit_update(self, kind: str, a, b, c=None, out_slots=None):
        """Submit an insert (a = src, b = dst, c = weights), delete (a = vertex,
        b = slot) or delete_pairs (a = u, b = v) batch; returns (ticket,
        out_slots) (slots filled for inserts)."""
        code = {"insert": OP_INSERT, "delete": OP_DELETE, "delete_pairs": OP_DELETE_PAIRS}.get(kind)
        if code is None:
            raise ValueError(f"unknown update kind {kind!r}")
        k = len(a) if not hasattr(a, "numel") else a.numel()
        pa, ka = _u32(a)
        pb, kb = _u32(b)
        pc, kc = _u32(c) if c is not None else (None, None)
        if kind == "insert" and out_slots is None:
            out_slots = np.zeros(k, np.uint32)
        po = _out(out_slots, np.uint32)[0] if out_slots is not None else None
        t = ctypes.c_uint64()
        self._check(self._L.bingo_serve_submit_update(self._h, code, pa, pb, pc, k, po, ctypes.byref(t)))
        self._serve_keep[t.value] = out_slots
        return t.value, out_slots

    @staticmethod
    def _status(s: BingoServeStatus) -> dict:
        return {"done": bool(s.done), "status": s.status, "kind": s.kind, "version": s.version,
                "latency_ns": s.latency_ns, "ready_ns": s.ready_ns}

    def serve_poll(self, ticket: int) -> dict:
        """Status of a serving ticket without waiting: done flag, request status,
        kind, graph version, latency and ready time."""
        s = BingoServeStatus()
        self._check(self._L.bingo_serve_poll(self._h, ticket, ctypes.byref(s)))
        return self._status(s)

    def serve_wait(self, ticket: int, timeout_us: int = 20_000_000) -> dict:
        """Wait for a ticket (bounded); raises BingoError(TIMEOUT) if it is not done in time."""
        s = BingoServeStatus()
        self._check(self._L.bingo_serve_wait(self._h, ticket, timeout_us, ctypes.byref(s)))
        self._serve_keep.pop(ticket, None)
        return self._status(s)

    # ------------------------------------------------------------ snapshots
    def save(self, path):
        """Write the whole graph store to a file (bingo_save)."""
        self._check(self._L.bingo_save(self._h, os.fsencode(path)))

    def restore(self, path):
        """Replace this handle's graph with a saved one (bingo_restore)."""
        self._check(self._L.bingo_restore(self._h, os.fsencode(path)))
        self.n = self.stats()["n"]

    # ------------------------------------------------------------ store check
    def check(self, raise_on_corrupt: bool = True) -> dict:
        """Verify every structural invariant of the graph store on the device
        (bingo_check): extents, live and group counts, group members and
        back-pointers, exact alias tables, the adjacency index, neighbour
        ranges. Returns the report; a failing store raises
        BingoError(BINGO_ERR_CORRUPT) unless raise_on_corrupt is false."""
        r = BingoCheckReport()
        st = self._L.bingo_check(self._h, ctypes.byref(r))
        rep = {f: getattr(r, f) for f, _ in BingoCheckReport._fields_}
        rep["kind_names"] = [name for bit, name in CHECK_KINDS.items() if r.kinds & bit]
        if st and not (st == 12 and not raise_on_corrupt):
            self._check(st)
        return rep

    # ------------------------------------------------------------ tuning
    def tuning(self) -> dict:
        """Current launch / batching knobs (bingo_get_tuning)."""
        t = BingoTuning()
        self._check(self._L.bingo_get_tuning(self._h, ctypes.byref(t)))
        return {f: getattr(t, f) for f in TUNING_FIELDS}

    def set_tuning(self, **knobs):
        """Change some knobs, keeping the others (bingo_set_tuning)."""
        cur = self.tuning()
        unknown = set(knobs) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning knobs {sorted(unknown)}")
        cur.update(knobs)
        t = BingoTuning(*[cur[f] for f in TUNING_FIELDS])
        self._check(self._L.bingo_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, jobs: Sequence[WalkJob] = (), inserts=None, deletes=None, repeats: int = 3,
                 cache: Optional[str] = None) -> dict:
        """Time the sample workload under candidate knobs and keep the fastest
        (bingo_autotune). inserts = (src, dst, w), deletes = (u, slot); the
        update sample is undone, so the graph is unchanged.

        cache: a JSON file of tuned knobs keyed by GPU model and workload shape
        (n, live edges, the jobs' apps / lengths / sizes, the update sizes);
        a hit sets the stored knobs without timing anything ("cached": True)."""
        key = None
        if cache is not None:
            key = self._tuning_key(jobs, inserts, deletes)
            table = _read_json(cache)
            if key in table:
                self.set_tuning(**table[key])
                return {"best": self.tuning(), "cached": True, "candidates": 0}
        rep = self._autotune(jobs, inserts, deletes, repeats)
        if cache is not None:
            table = _read_json(cache)
            table[key] = rep["best"]
            tmp = f"{cache}.tmp{os.getpid()}"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        rep["cached"] = False
        return rep

    def _tuning_key(self, jobs, inserts, deletes) -> str:
        import torch
        st = self.stats()
        size = lambda a: 0 if a is None else (a[0].numel() if hasattr(a[0], "numel") else len(a[0]))  # noqa: E731
        shape = [(j.app, j.length, j.n_starts if j.starts is None else
                  (j.starts.numel() if hasattr(j.starts, "numel") else len(j.starts))) for j in jobs]
        return json.dumps([torch.cuda.get_device_name(self.device), st["n"], st["live_edges"], shape,
                           size(inserts), size(deletes)])

    def _autotune(self, jobs, inserts, deletes, repeats) -> dict:
        keep = []
        req = BingoTuneRequest()
        if jobs:
            arr = self._job_array(list(jobs), keep)
            keep.append(arr)
            req.jobs = ctypes.cast(arr, ctypes.c_void_p)
            req.n_jobs = len(jobs)
        req.repeats = repeats
        if inserts is not None:
            cols = [_u32(x) for x in inserts]
            keep += [c[1] for c in cols]
            req.ins_src, req.ins_dst, req.ins_w = (c[0] for c in cols)
            req.n_ins = len(inserts[0]) if not hasattr(inserts[0], "numel") else inserts[0].numel()
        if deletes is not None:
            cols = [_u32(x) for x in deletes]
            keep += [c[1] for c in cols]
            req.del_u, req.del_slot = (c[0] for c in cols)
            req.n_del = len(deletes[0]) if not hasattr(deletes[0], "numel") else deletes[0].numel()
        rep = BingoTuneReport()
        self._check(self._L.bingo_autotune(self._h, ctypes.byref(req), ctypes.byref(rep)))
        out = {f: getattr(rep, f) for f, _ in BingoTuneReport._fields_ if f not in ("best", "reserved0")}
        out["best"] = {f: getattr(rep.best, f) for f in TUNING_FIELDS}
        return out

    def serve_metrics(self) -> dict:
        """Serving counters: submitted and completed requests, walk-kernel launches,
        scheduler time per phase (admission, completion, updates, drain waits) and
        the summed queue, device and copy time of walk queries."""
        m = BingoServeMetrics()
        self._check(self._L.bingo_serve_get_metrics(self._h, ctypes.byref(m)))
        return {f: getattr(m, f) for f, _ in BingoServeMetrics._fields_}

    def serve_stop(self):
        """Finish every submitted request, stop the walk loop and return the handle to normal use."""
        self._check(self._L.bingo_serve_stop(self._h))
        self._serve_keep = {}

    def sync(self):
        """Wait for all queued work; raises the first device-detected error since the last sync."""
        self._check(self._L.bingo_sync(self._h))

    def set_stream(self, stream_ptr: int):
        """Order later calls on a caller's CUDA stream (its handle as an int, e.g.
        torch.cuda.Stream().cuda_stream); 0 restores the handle's own stream."""
        self._check(self._L.bingo_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def stats(self) -> dict:
        """Counts (vertices, slots, live edges), arena and scratch bytes, walk steps,
        kernel launches and node2vec proposals / adjacency probes since creation."""
        s = BingoStats()
        self._check(self._L.bingo_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in BingoStats._fields_ if f != "reserved0"}

    def dump(self) -> dict:
        """Full graph state in the layout the CPU oracle dumps (numpy arrays)."""
        sizes = (ctypes.c_uint64 * 3)()
        self._check(self._L.bingo_dump_sizes(self._h, sizes))
        ns, nm, na = sizes[0], sizes[1], sizes[2]
        n = self.n
        d = dict(
            ecnt=np.zeros(n, np.uint32), live=np.zeros(n, np.uint32), ev=np.zeros(ns, np.uint32),
            ew=np.zeros(ns, np.uint32), gcnt=np.zeros(n * 32, np.uint32), mslot=np.zeros(nm, np.uint32),
            mv=np.zeros(nm, np.uint32), mbp=np.zeros(nm, np.uint32), am=np.zeros(n, np.uint32),
            athr=np.zeros(na, np.uint64), aT=np.zeros(na, np.uint64), aown=np.zeros(na, np.uint8),
            aalias=np.zeros(na, np.uint8))
        order = ["ecnt", "live", "ev", "ew", "gcnt", "mslot", "mv", "mbp", "am", "athr", "aT", "aown", "aalias"]
        ptrs = [ctypes.c_void_p(d[k].ctypes.data) for k in order]
        self._check(self._L.bingo_dump_state(self._h, *ptrs))
        return d

    def philox(self, ctr: np.ndarray, key: int) -> np.ndarray:
        """Philox4x32-10 blocks as the walk kernels compute them: one row of four
        words out per row of four counter words in, under the 64-bit key."""
        ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
        out = np.zeros_like(ctr)
        self._check(self._L.bingo_philox(self._h, ctypes.c_void_p(ctr.ctypes.data), ctr.shape[0], key,
                                         ctypes.c_void_p(out.ctypes.data)))
        return out

    def probe_gather(self, table_bytes: int = 4 << 30) -> dict:
        """Random 32-byte-sector read rates of this GPU (independent and
        dependent-chain forms) and the dependent-read latency."""
        out = np.zeros(3, np.float64)
        self._check(self._L.bingo_probe_gather(self._h, table_bytes, ctypes.c_void_p(out.ctypes.data)))
        return {"independent_sectors_per_s": float(out[0]), "chain_sectors_per_s": float(out[1]),
                "chain_latency_ns": float(out[2]), "table_bytes": table_bytes}

    # ---------------------------------------------- reference-named aliases
    def build(self, src, dst, w, n: int):
        """Alias of load_edges under the reference's name (include/operation.cuh:33)."""
        return self.load_edges(src, dst, w, n)

    def insert(self, src, dst, w):
        """Alias of insert_batch under the reference's name (include/operation.cuh:144)."""
        return self.insert_batch(src, dst, w)

    def deleteE(self, u, slot):
        """Alias of delete_batch under the reference's name (include/operation.cuh:215)."""
        return self.delete_batch(u, slot)
