"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs. Graph state (slots, tombstones, group member sequences,
back-pointers, alias tables) and walks must be bit-exact."""
import glob
import os

import numpy as np
import pytest

from bingo_b200 import BATCHED, DEEPWALK, NODE2VEC, PLAIN, PPR, SAMPLING, WALK_PPR_TAIL, BingoError, Graph, WalkJob, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, check_exact_invariants, workload

pytestmark = pytest.mark.gpu


def replay(n, src, dst, w, ops, check_every=True, **gkw):
    g = Graph(**gkw)
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    assert_exact_equal(g.dump(), ex.dump(), "load: ")
    for i, op in enumerate(ops):
        if op[0] == "ins":
            s_gpu = g.insert_batch(*op[1:])
            s_ora = ex.insert(*op[1:])
            assert np.array_equal(s_gpu, s_ora), f"op {i}: slot ids"
        else:
            g.delete_batch(*op[1:])
            assert ex.delete(*op[1:]) == 0
        if check_every or i == len(ops) - 1:
            d = g.dump()
            assert_exact_equal(d, ex.dump(), f"op {i} ({op[0]}): ")
    check_exact_invariants(g.dump(), n)
    return g, ex


@pytest.mark.parametrize("dist,lo,hi", [(gen.W_UNIFORM, 1, 1024), (gen.W_LOGUNIFORM, 1, 2 ** 20),
                                        (gen.W_ZIPF, 1, 2 ** 24 - 1), (gen.W_UNIFORM, 1, 2 ** 32 - 1)])
def test_state_parity_small(dist, lo, hi):
    n, src, dst, w, ops = workload(scale=10, ef=16, seed=17, dist=dist, lo=lo, hi=hi, rounds=3, k_ins=700,
                                   k_del=700)
    replay(n, src, dst, w, ops)


def test_state_parity_rmat14():
    """The small DeepWalk workload: R-MAT 14 / ef 16, uniform [1,1024], 10K + 10K."""
    n, src, dst, w, ops = workload(scale=14, ef=16, seed=1235, rounds=1, k_ins=10000, k_del=10000)
    replay(n, src, dst, w, ops)


def test_state_parity_growth_paths():
    """Tiny arenas force every relocation path (edges, back-pointers, groups,
    alias, adjacency) and host-side arena regrowth."""
    n, src, dst, w, ops = workload(scale=9, ef=4, seed=23, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 31, rounds=4,
                                   k_ins=3000, k_del=500)
    g, _ = replay(n, src, dst, w, ops, arena_factor=1.0)
    st = g.stats()
    assert st["arena_used"] <= st["arena_bytes"]


def test_hub_vertex_batches():
    """Many inserts to one vertex in one batch (long segments, multi-chunk ballots)."""
    n = 4096
    src = np.zeros(5000, np.uint32)
    dst = (np.arange(5000) % (n - 1) + 1).astype(np.uint32)
    w = gen.weights(5000, gen.W_LOGUNIFORM, 1, 2 ** 30, seed=3)
    ins_src = np.concatenate([np.zeros(7000, np.uint32), np.full(100, 5, np.uint32)])
    ins_dst = (np.arange(7100) % (n - 2) + 2).astype(np.uint32)
    ins_w = gen.weights(7100, gen.W_UNIFORM, 1, 2 ** 32 - 1, seed=4)
    dels = np.arange(0, 12000, 3, dtype=np.uint32)
    ops = [("ins", ins_src, ins_dst, ins_w), ("del", np.zeros(len(dels), np.uint32), dels)]
    replay(n, src, dst, w, ops)


def _walk_both(g, ex, n, app, L, starts, mode, **kw):
    out = g.walk(app=app, length=L, starts=starts, mode=mode, **kw)
    ref = ex.walk(app, L, starts, seed=kw.get("seed", 0), job_id=kw.get("job_id", 0), p=kw.get("p", 0.5),
                  q=kw.get("q", 2.0), stop=kw.get("stop_prob", 0.0125), flags=kw.get("flags", 0))
    return out, ref


@pytest.fixture(scope="module")
def rmat14_graphs():
    n, src, dst, w, ops = workload(scale=14, ef=16, seed=1235, rounds=1, k_ins=10000, k_del=10000)
    g = Graph()
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    return n, g, ex, ops


@pytest.mark.parametrize("mode", [PLAIN, BATCHED])
@pytest.mark.parametrize("app,kw", [(DEEPWALK, {}), (NODE2VEC, dict(p=0.5, q=2.0)), (NODE2VEC, dict(p=4.0, q=0.25)),
                                    (PPR, dict(stop_prob=0.15)), (PPR, dict(stop_prob=0.0125, flags=WALK_PPR_TAIL)),
                                    (SAMPLING, {})])
def test_walk_parity(rmat14_graphs, app, kw, mode):
    n, g, ex, _ = rmat14_graphs
    starts = np.arange(n, dtype=np.uint32)
    out, ref = _walk_both(g, ex, n, app, 80, starts, mode, seed=0xB1460 + app, job_id=3, **kw)
    assert np.array_equal(out, ref)


def test_walk_parity_after_updates():
    n, src, dst, w, ops = workload(scale=14, ef=16, seed=1235, rounds=1, k_ins=10000, k_del=10000)
    g, ex = replay(n, src, dst, w, ops, check_every=False)
    starts = np.arange(n, dtype=np.uint32)
    for app in (DEEPWALK, NODE2VEC, PPR):
        out, ref = _walk_both(g, ex, n, app, 80, starts, PLAIN, seed=77, job_id=app)
        assert np.array_equal(out, ref), app


def test_batched_heterogeneous_jobs(rmat14_graphs):
    n, g, ex, _ = rmat14_graphs
    rng = np.random.default_rng(0)
    jobs, refs = [], []
    specs = [(DEEPWALK, 10, {}), (NODE2VEC, 37, dict(p=0.25, q=4.0)), (PPR, 200, dict(stop_prob=0.15)),
             (SAMPLING, 1, {}), (DEEPWALK, 5, {}), (NODE2VEC, 80, dict(p=1.0, q=1.0))]
    for jid, (app, L, kw) in enumerate(specs):
        starts = rng.integers(0, n, size=int(rng.integers(1, 3000)), dtype=np.uint32)
        out = np.zeros(len(starts) if app == SAMPLING else (len(starts), L), np.int32)
        jobs.append(WalkJob(app=app, length=L, starts=starts, n_starts=len(starts), seed=99, job_id=jid, out=out,
                            **kw))
        refs.append(ex.walk(app, L, starts, seed=99, job_id=jid, p=kw.get("p", 0.5), q=kw.get("q", 2.0),
                            stop=kw.get("stop_prob", 0.0125)))
    g.walk_jobs(jobs, mode=BATCHED)
    for j, r in zip(jobs, refs):
        assert np.array_equal(j.out, r)
    for j in jobs:
        j.out[...] = 0
    g.walk_jobs(jobs, mode=PLAIN)
    for j, r in zip(jobs, refs):
        assert np.array_equal(j.out, r)


def test_walk_range_and_empty(rmat14_graphs):
    n, g, ex, _ = rmat14_graphs
    out = g.walk(app=DEEPWALK, length=80, first=100, n_starts=500, seed=5)
    ref = ex.walk(DEEPWALK, 80, np.arange(100, 600, dtype=np.uint32), seed=5)
    assert np.array_equal(out, ref)
    z = g.walk(app=DEEPWALK, length=80, starts=np.zeros(0, np.uint32), seed=5)
    assert z.shape == (0, 80)
    one = g.walk(app=DEEPWALK, length=1, starts=np.arange(10, dtype=np.uint32))
    assert np.array_equal(one[:, 0], np.arange(10))


def test_device_tensors(rmat14_graphs):
    torch = pytest.importorskip("torch")
    n, g, ex, _ = rmat14_graphs
    starts = torch.arange(0, n, dtype=torch.int32, device="cuda")
    out = torch.empty((n, 40), dtype=torch.int32, device="cuda")
    g.walk(app=DEEPWALK, length=40, starts=starts, out=out, seed=12)
    ref = ex.walk(DEEPWALK, 40, np.arange(n, dtype=np.uint32), seed=12)
    assert np.array_equal(out.cpu().numpy(), ref)


def test_device_tensor_updates():
    torch = pytest.importorskip("torch")
    n, src, dst, w, ops = workload(scale=10, ef=8, seed=31, rounds=1, k_ins=300, k_del=300)
    g = Graph()
    ex = po.ExactGraph(n)
    t = lambda a: torch.from_numpy(a.astype(np.int32)).cuda()  # noqa: E731
    g.load_edges(t(src), t(dst), t(w), n)
    ex.load(src, dst, w)
    ins = ops[0]
    slots = torch.empty(len(ins[1]), dtype=torch.int32, device="cuda")
    g.insert_batch(t(ins[1]), t(ins[2]), t(ins[3]), out_slots=slots)
    assert np.array_equal(slots.cpu().numpy().astype(np.uint32), ex.insert(*ins[1:]))
    g.delete_batch(t(ops[1][1]), t(ops[1][2]))
    ex.delete(*ops[1][1:])
    assert_exact_equal(g.dump(), ex.dump())


def test_errors_leave_state_unchanged():
    n, src, dst, w, ops = workload(scale=8, ef=8, seed=41, rounds=1, k_ins=50, k_del=50)
    g = Graph()
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    before = g.dump()
    with pytest.raises(BingoError) as e:
        g.insert_batch([1, 2], [3, n], [1, 1])
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    with pytest.raises(BingoError) as e:
        g.insert_batch([1, 2], [3, 4], [1, 0])
    assert e.value.name == "BINGO_ERR_ZERO_WEIGHT"
    with pytest.raises(BingoError) as e:
        g.delete_batch([n + 5], [0])
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    assert_exact_equal(g.dump(), before)
    # absent and repeated slots are skipped; the valid deletes still apply
    u0 = int(src[0])
    with pytest.raises(BingoError) as e:
        g.delete_batch([u0, u0, u0], [0, 0, 10 ** 6])
    assert e.value.name == "BINGO_ERR_INVALID_SLOT"
    assert ex.delete([u0, u0, u0], [0, 0, 10 ** 6]) == 2
    assert_exact_equal(g.dump(), ex.dump())
    with pytest.raises(BingoError) as e:
        g.walk(app=DEEPWALK, length=10, starts=[n])
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    g2 = Graph(node2vec=False)
    g2.load_edges(src, dst, w, n)
    with pytest.raises(BingoError) as e:
        g2.walk(app=NODE2VEC, length=10, starts=[0])
    assert e.value.name == "BINGO_ERR_UNSUPPORTED"
    with pytest.raises(BingoError) as e:
        Graph().walk(app=DEEPWALK, length=10, starts=[0])
    assert e.value.name == "BINGO_ERR_NOT_LOADED"


def test_device_side_validation():
    """Out-of-range ids in device-resident batches are caught on the device;
    the batch is not applied."""
    torch = pytest.importorskip("torch")
    n, src, dst, w, _ = workload(scale=8, ef=8, seed=43, rounds=0)
    g = Graph()
    g.load_edges(src, dst, w, n)
    before = g.dump()
    bad = torch.tensor([1, n + 3], dtype=torch.int32, device="cuda")
    ok = torch.tensor([2, 3], dtype=torch.int32, device="cuda")
    one = torch.tensor([1, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(BingoError) as e:
        g.insert_batch(bad, ok, one)
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    with pytest.raises(BingoError) as e:
        g.insert_batch(ok, ok, torch.tensor([1, 0], dtype=torch.int32, device="cuda"))
    assert e.value.name == "BINGO_ERR_ZERO_WEIGHT"
    assert_exact_equal(g.dump(), before)


def test_philox_matches_oracle():
    g = Graph()
    rng = np.random.default_rng(1)
    ctr = rng.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    key = 0x0123456789ABCDEF
    out = g.philox(ctr, key)
    for i in range(0, 4096, 97):
        assert list(out[i]) == list(po.philox(ctr[i], [key & 0xFFFFFFFF, key >> 32]))


def test_multi_edges_and_reload():
    """Duplicate (u, v) pairs are separate slots; reloading replaces the graph."""
    n = 16
    src = np.array([0, 0, 0, 1, 1], np.uint32)
    dst = np.array([1, 1, 2, 0, 0], np.uint32)
    w = np.array([3, 5, 7, 1, 2], np.uint32)
    ops = [("ins", np.array([0, 0], np.uint32), np.array([1, 3], np.uint32), np.array([9, 1], np.uint32)),
           ("del", np.array([0, 1], np.uint32), np.array([1, 0], np.uint32))]
    g, ex = replay(n, src, dst, w, ops)
    g.load_edges(src[:2], dst[:2], w[:2], 4)
    ex2 = po.ExactGraph(4)
    ex2.load(src[:2], dst[:2], w[:2])
    assert_exact_equal(g.dump(), ex2.dump())


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz"))),
                         ids=os.path.basename)
def test_cuda_state_matches_reference_binary(path):
    """The CUDA path against the reference's own CUDA build: after the load
    and after every batch, every list the reference keeps (sparse groups in
    member order, back-pointers), the float masses below its load-time bit
    length, slots, weights and tombstones equal the reference's dump."""
    import json
    from tests.helpers import compare_exact_vs_ref
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    n = meta["n"]
    g = Graph()
    g.load_edges(z["src"], z["dst"], z["w"], n)
    names = ["logt", "bits", "sz", "ecnt", "asz", "ev", "ew", "grouptp", "num", "gsz", "members", "midx", "ap",
             "aa", "ab"]
    for i, op in enumerate(["load"] + meta["ops"]):
        if op == "ins":
            g.insert_batch(z[f"op{i}_a"], z[f"op{i}_b"], z[f"op{i}_c"])
        elif op == "del":
            g.delete_batch(z[f"op{i}_a"], z[f"op{i}_b"])
        ref = {k: z[f"dump{i}_{k}"] for k in names}
        compare_exact_vs_ref(g.dump(), ref, n, check_alias_tol=5e-3)


def test_group_lists_shrink_and_regrow(tmp_path):
    """Group capacity is derived from the count plus a hysteresis bit: a list
    whose count dips below a power of two and climbs back keeps its storage
    (no move per cycle), a deep dip followed by regrowth moves it, and the
    state stays equal to the oracle's throughout."""
    from tests.test_gpu_check import Snap
    n = 64
    src = np.zeros(20, np.uint32)
    dst = np.arange(1, 21, dtype=np.uint32)
    w = np.ones(20, np.uint32)  # every edge in group 0 only: its count is vertex 0's degree
    src = np.concatenate([src, np.arange(1, 40, dtype=np.uint32)])
    dst = np.concatenate([dst, np.arange(2, 41, dtype=np.uint32)])
    w = np.concatenate([w, gen.weights(39, gen.W_UNIFORM, 1, 1000, seed=7)])
    g, ex = Graph(node2vec=True), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    live = list(range(20))  # live slots of vertex 0

    def group0():
        p = tmp_path / "s.snap"
        g.save(p)
        return Snap(p.read_bytes()).group(0, 0)

    def cycle(k, seed):
        rng = np.random.default_rng(seed)
        pick = sorted(rng.choice(len(live), size=k, replace=False).tolist(), reverse=True)
        slots = np.array([live.pop(i) for i in pick], np.uint32)
        u = np.zeros(k, np.uint32)
        g.delete_batch(u, slots)
        assert ex.delete(u, slots) == 0
        assert_exact_equal(g.dump(), ex.dump(), f"after deleting {k}: ")
        v = rng.integers(1, n, size=k).astype(np.uint32)
        ins = (u, v, np.ones(k, np.uint32))
        got = g.insert_batch(*ins)
        assert np.array_equal(got, ex.insert(*ins))
        live.extend(got.tolist())
        assert_exact_equal(g.dump(), ex.dump(), f"after reinserting {k}: ")

    base0, cnt0, cap0 = group0()
    assert cnt0 == 20 and cap0 == 32
    for c in range(6):  # 20 -> 15 -> 20: below 16 and back, within the list's 32 entries
        cycle(5, 100 + c)
        base, cnt, cap = group0()
        assert (base, cnt) == (base0, 20), f"cycle {c}: the list moved ({base0} -> {base})"
    for c in range(3):  # 20 -> 3 -> 20: the deep dip forgets the spare room, regrowth moves the list
        cycle(17, 200 + c)
        assert group0()[1] == 20
    assert g.check()["bad_vertices"] == 0
    walks = g.walk(app=DEEPWALK, length=30, starts=np.arange(n, dtype=np.uint32), seed=3)
    assert np.array_equal(walks, ex.walk(DEEPWALK, 30, np.arange(n, dtype=np.uint32), seed=3))
