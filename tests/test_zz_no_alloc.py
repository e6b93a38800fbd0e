"""bingo_walk_noalloc: walks for callers that cannot call cudaMalloc while
they run (a serving loop whose HBM is budgeted to the graph and its outputs,
an application that owns the device memory pool). The entry point takes its
scratch from a fixed array in the library. Checked through the C ABI against
the allocating entry point, bingo_walk(BATCHED), bit for bit, on two calls in
a row, and checked to leave the handle's device memory and the device's free
memory unchanged. This file is collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs(torch, n, call):
    from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING
    rng = np.random.default_rng(100 + call)
    specs = [(DEEPWALK, 80, {}), (NODE2VEC, 40, dict(p=0.5, q=2.0)), (PPR, 80, dict(stop_prob=0.15)),
             (SAMPLING, 1, {}), (DEEPWALK, 7, {}), (NODE2VEC, 25, dict(p=4.0, q=0.25))]
    out = []
    for jid, (app, L, kw) in enumerate(specs):
        k = int(rng.integers(100, 5000))
        starts = torch.from_numpy(rng.integers(0, n, size=k).astype(np.int32)).cuda()
        shape = (k,) if app == SAMPLING else (k, L)
        out.append(dict(app=app, length=L, starts=starts, n_starts=k, seed=7 + call, job_id=jid,
                        p=kw.get("p", 0.5), q=kw.get("q", 2.0), stop_prob=kw.get("stop_prob", 0.0125),
                        a=torch.full(shape, -7, dtype=torch.int32, device="cuda"),
                        b=torch.full(shape, -9, dtype=torch.int32, device="cuda")))
    # one range job (starts = NULL)
    out.append(dict(app=DEEPWALK, length=16, starts=None, n_starts=n // 2, seed=11 + call, job_id=99, p=0.5,
                    q=2.0, stop_prob=0.0, a=torch.full((n // 2, 16), -7, dtype=torch.int32, device="cuda"),
                    b=torch.full((n // 2, 16), -9, dtype=torch.int32, device="cuda")))
    return out


def _abi_jobs(specs, key):
    from bingo_b200._lib import BingoWalkJob
    arr = (BingoWalkJob * len(specs))()
    for i, s in enumerate(specs):
        arr[i].app = s["app"]
        arr[i].length = s["length"]
        arr[i].starts = ctypes.c_void_p(s["starts"].data_ptr()) if s["starts"] is not None else None
        arr[i].n_starts = s["n_starts"]
        arr[i].first = 0
        arr[i].job_id = s["job_id"]
        arr[i].seed = s["seed"]
        arr[i].flags = 0
        arr[i].p, arr[i].q, arr[i].stop_prob = s["p"], s["q"], s["stop_prob"]
        arr[i].out = ctypes.c_void_p(s[key].data_ptr())
    return arr


def test_noalloc_walks_match_allocating_entry_point():
    torch = pytest.importorskip("torch")
    from bingo_b200 import BATCHED, Graph, gen
    from bingo_b200._lib import lib
    L = lib()
    n = 1 << 12
    src, dst = gen.rmat(12, 16, seed=91)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 20, seed=92)
    g = Graph()
    g.load_edges(src, dst, w, n)
    for call in range(2):
        specs = _jobs(torch, n, call)
        ref = _abi_jobs(specs, "a")
        assert L.bingo_walk(g.handle, ref, len(specs), BATCHED) == 0, L.bingo_last_error(g.handle)
        mine = _abi_jobs(specs, "b")
        torch.cuda.synchronize()
        held = _held(g)
        free0 = torch.cuda.mem_get_info()[0]
        st = L.bingo_walk_noalloc(g.handle, mine, len(specs))
        assert st == 0, L.bingo_last_error(g.handle)
        torch.cuda.synchronize()
        # The handle holds no more device memory than before the call.
        assert _held(g) == held, (call, held, _held(g))
        if call == 1:
            # After the first call (which may load the kernels it launches),
            # the device's free memory does not move either.
            assert torch.cuda.mem_get_info()[0] == free0
        for s in specs:
            assert torch.equal(s["a"], s["b"]), f"call {call} job {s['job_id']}"
            assert (s["b"] != -9).all()


def _held(g):
    st = g.stats()
    return st["scratch_bytes"], st["arena_bytes"]


def test_noalloc_rejects_what_it_cannot_do_without_allocating():
    torch = pytest.importorskip("torch")
    from bingo_b200 import Graph, gen
    from bingo_b200._lib import BingoWalkJob, lib
    L = lib()
    n = 1 << 10
    src, dst = gen.rmat(10, 8, seed=93)
    g = Graph()
    g.load_edges(src, dst, gen.weights(len(src), seed=94), n)
    out = torch.zeros((4, 8), dtype=torch.int32, device="cuda")
    many = (BingoWalkJob * 65)()
    for j in many:
        j.app, j.length, j.n_starts, j.out = 0, 8, 4, ctypes.c_void_p(out.data_ptr())
    assert L.bingo_walk_noalloc(g.handle, many, 65) == 1
    assert b"at most 64 jobs" in L.bingo_last_error(g.handle)
    host_out = np.zeros((4, 8), np.int32)
    one = (BingoWalkJob * 1)()
    one[0].app, one[0].length, one[0].n_starts = 0, 8, 4
    one[0].out = ctypes.c_void_p(host_out.ctypes.data)
    assert L.bingo_walk_noalloc(g.handle, one, 1) == 1
    assert b"device output" in L.bingo_last_error(g.handle)
