"""Serving: walk queries admitted into a running device loop (continuous
batching) with update batches interleaved. Every query's rows must equal the
same query run alone on the graph version it saw (the updates submitted
before it), checked against the CPU oracle replaying the stream in order."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING, BingoError, Graph, gen
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _graph(scale=11, seed=81):
    n = 1 << scale
    src, dst = gen.rmat(scale, 16, seed=seed)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 65535, seed=seed + 1)
    return n, src, dst, w


def test_served_results_equal_alone_results():
    n, src, dst, w = _graph()
    g = Graph()
    g.load_edges(src, dst, w, n)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=85)
    rng = np.random.default_rng(86)
    g.serve_start(output_budget_bytes=64 << 20, idle_timeout_us=500)
    trace = []
    apps = [(DEEPWALK, 80, {}), (PPR, 80, dict(stop_prob=0.15)), (NODE2VEC, 40, dict(p=0.5, q=2.0)),
            (SAMPLING, 1, {})]
    for r in range(60):
        if r % 7 == 6:
            if r % 2:
                ins = ug.inserts(int(rng.integers(1, 800)), gen.W_UNIFORM, 1, 65535)
                t, slots = g.submit_update("insert", *ins)
                trace.append(("insert", t, ins, slots))
            else:
                dels = ug.deletes(int(rng.integers(1, 800)))
                t, _ = g.submit_update("delete", *dels)
                trace.append(("delete", t, dels))
        else:
            app, L, kw = apps[r % len(apps)]
            starts = rng.integers(0, n, size=int(rng.integers(1, 3000))).astype(np.uint32)
            t, out = g.submit_walk(app=app, length=L, starts=starts, seed=1000 + r, job_id=r, **kw)
            trace.append(("walk", t, (app, L, starts, r, kw), out))
    results = {}
    for item in trace:
        results[item[1]] = g.serve_wait(item[1])
    g.serve_stop()
    version = 0
    for item in trace:
        st = results[item[1]]
        assert st["done"] and st["status"] == 0, st
        if item[0] == "walk":
            app, L, starts, r, kw = item[2]
            assert st["version"] == version
            ref = ex.walk(app, L, starts, seed=1000 + r, job_id=r, p=kw.get("p", 0.5), q=kw.get("q", 2.0),
                          stop=kw.get("stop_prob", 0.0125))
            assert np.array_equal(item[3], ref), f"query {r} (app {app}) differs from its solo run"
        elif item[0] == "insert":
            version += 1
            assert np.array_equal(item[3], ex.insert(*item[2]))
        else:
            version += 1
            assert ex.delete(*item[2]) == 0
    from tests.helpers import assert_exact_equal
    assert_exact_equal(g.dump(), ex.dump())


def test_continuous_batching_shares_launches():
    """Many queries submitted back to back run inside a few walk-loop launches."""
    n, src, dst, w = _graph(scale=12, seed=91)
    g = Graph()
    g.load_edges(src, dst, w, n)
    g.serve_start(idle_timeout_us=20000)
    l0 = g.stats()["kernel_launches"]
    rng = np.random.default_rng(92)
    tickets = [g.submit_walk(app=DEEPWALK, length=60, starts=rng.integers(0, n, size=500).astype(np.uint32),
                             seed=i, job_id=i)[0] for i in range(200)]
    for t in tickets:
        assert g.serve_wait(t)["status"] == 0
    launches = g.stats()["kernel_launches"] - l0
    g.serve_stop()
    assert launches <= 20, launches


def test_admission_by_budget_and_busy_guard():
    n, src, dst, w = _graph(scale=10, seed=95)
    g = Graph()
    g.load_edges(src, dst, w, n)
    g.serve_start(output_budget_bytes=1 << 20)  # 1 MiB: a 5000 x 80 query needs 1.6 MB
    with pytest.raises(BingoError) as e:
        g.submit_walk(app=DEEPWALK, length=80, starts=np.zeros(5000, np.uint32))
    assert e.value.name == "BINGO_ERR_CAPACITY"
    # queries that fit one at a time are admitted as memory frees up
    tickets = [g.submit_walk(app=DEEPWALK, length=80, starts=np.full(2000, i, np.uint32), seed=i, job_id=i)
               for i in range(12)]
    with pytest.raises(BingoError) as e:
        g.walk(app=DEEPWALK, length=8, starts=[0])
    assert e.value.name == "BINGO_ERR_BUSY"
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    for i, (t, out) in enumerate(tickets):
        assert g.serve_wait(t)["status"] == 0
        assert np.array_equal(out, ex.walk(DEEPWALK, 80, np.full(2000, i, np.uint32), seed=i, job_id=i))
    g.serve_stop()
    g.walk(app=DEEPWALK, length=8, starts=[0])  # usable again


def test_stalled_producer_and_bad_update():
    """Failure handling without a GPU fault: when the producer stalls past the
    idle limit, the serving kernel's bounded wait ends and the kernel exits
    (the next query relaunches it and still gets exact rows); a malformed
    update fails only its own ticket."""
    import time
    n, src, dst, w = _graph(scale=11, seed=97)
    g = Graph()
    g.load_edges(src, dst, w, n)
    ref = Graph()
    ref.load_edges(src, dst, w, n)
    g.serve_start(idle_timeout_us=2000)
    rng = np.random.default_rng(98)
    st1 = rng.integers(0, n, size=300).astype(np.uint32)
    t, out1 = g.submit_walk(app=DEEPWALK, length=30, starts=st1, seed=1, job_id=1)
    assert g.serve_wait(t)["status"] == 0
    l1 = g.serve_metrics()["walk_kernel_launches"]
    time.sleep(0.05)  # the producer stalls for 25x the idle limit
    st2 = rng.integers(0, n, size=300).astype(np.uint32)
    t2, out2 = g.submit_walk(app=DEEPWALK, length=30, starts=st2, seed=2, job_id=2)
    assert g.serve_wait(t2)["status"] == 0
    # a still-running kernel would have taken this query without a launch
    assert g.serve_metrics()["walk_kernel_launches"] == l1 + 1
    bad = np.array([0, n + 7], np.uint32)
    tb, _ = g.submit_update("insert", bad, np.array([1, 2], np.uint32), np.array([3, 4], np.uint32))
    st3 = rng.integers(0, n, size=300).astype(np.uint32)
    t3, out3 = g.submit_walk(app=DEEPWALK, length=30, starts=st3, seed=3, job_id=3)
    assert g.serve_wait(tb)["status"] != 0  # OUT_OF_RANGE, nothing applied
    assert g.serve_wait(t3)["status"] == 0
    g.serve_stop()
    assert np.array_equal(out3, ref.walk(app=DEEPWALK, length=30, starts=st3, seed=3, job_id=3))
    assert np.array_equal(out1, ref.walk(app=DEEPWALK, length=30, starts=st1, seed=1, job_id=1))
    assert np.array_equal(out2, ref.walk(app=DEEPWALK, length=30, starts=st2, seed=2, job_id=2))
    assert g.stats()["live_edges"] == len(src)


def test_update_status_and_back_to_back_updates():
    """Updates commit without a host wait: a delete batch holding an absent
    slot (a repeated delete) reports BINGO_ERR_INVALID_SLOT on its own ticket
    once its valid deletes have applied; two updates submitted back to back
    apply in order; a query submitted right after them sees both, and the
    store ends equal to the oracle's."""
    n, src, dst, w = _graph(scale=11, seed=99)
    g = Graph()
    g.load_edges(src, dst, w, n)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=100)
    rng = np.random.default_rng(101)
    g.serve_start(idle_timeout_us=2000)
    warm = rng.integers(0, n, size=200).astype(np.uint32)
    t0, out0 = g.submit_walk(app=DEEPWALK, length=20, starts=warm, seed=5, job_id=5)
    ins = ug.inserts(500, gen.W_UNIFORM, 1, 65535)
    t1, slots = g.submit_update("insert", *ins)
    du, ds = ug.deletes(300)
    du = np.concatenate([du, du[:1]]).astype(np.uint32)  # the repeat is an absent slot: skipped, reported
    ds = np.concatenate([ds, ds[:1]]).astype(np.uint32)
    t2, _ = g.submit_update("delete", du, ds)
    starts = rng.integers(0, n, size=1500).astype(np.uint32)
    t3, out3 = g.submit_walk(app=PPR, length=40, starts=starts, seed=6, job_id=6, stop_prob=0.15)
    s0, s1, s2, s3 = (g.serve_wait(t) for t in (t0, t1, t2, t3))
    g.serve_stop()
    assert s0["status"] == 0 and s0["version"] == 0
    assert s1["status"] == 0 and s1["version"] == 1
    assert s2["status"] == 4 and s2["version"] == 2  # BINGO_ERR_INVALID_SLOT
    assert s3["status"] == 0 and s3["version"] == 2
    assert np.array_equal(out0, ex.walk(DEEPWALK, 20, warm, seed=5, job_id=5))
    assert np.array_equal(slots, ex.insert(*ins))
    assert ex.delete(du, ds) == 1
    assert np.array_equal(out3, ex.walk(PPR, 40, starts, seed=6, job_id=6, stop=0.15))
    from tests.helpers import assert_exact_equal
    assert_exact_equal(g.dump(), ex.dump())
