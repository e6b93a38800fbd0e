"""Edge cases against the oracle, bit for bit: a vertex without out-edges at
load becomes walkable once edges arrive (the reference never walks from it,
include/Bingo.cuh:186), a vertex whose every edge is deleted becomes a dead
end and revives on re-insert, extreme weights, self-loops, and an empty
graph that grows."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING, Graph
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, check_exact_invariants

pytestmark = pytest.mark.gpu

U = lambda *x: np.array(x, np.uint32)  # noqa: E731


def _pair(n, node2vec=True):
    return Graph(node2vec=node2vec), po.ExactGraph(n)


def _walks_equal(g, ex, starts, length=12, seed=3):
    for app in (DEEPWALK, NODE2VEC, PPR, SAMPLING):
        a = g.walk(app=app, length=length, starts=starts, seed=seed, job_id=app, stop_prob=0.3)
        b = ex.walk(app, length, starts, seed=seed, job_id=app, stop=0.3)
        assert np.array_equal(a, b), app
    return g.walk(app=DEEPWALK, length=length, starts=starts, seed=seed)


def test_dead_end_revival_and_full_deletion():
    n = 8
    g, ex = _pair(n)
    src, dst, w = U(0, 0, 0, 2, 3), U(1, 2, 3, 0, 0), U(5, 9, 1 << 20, 7, 3)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    starts = np.arange(n, dtype=np.uint32)
    rows = _walks_equal(g, ex, starts)
    assert (rows[1, 1:] == -1).all()  # vertex 1 has no out-edge yet
    # vertex 1 gains edges: it walks now
    s = g.insert_batch(U(1, 1), U(4, 0), U(2, 6))
    assert np.array_equal(s, ex.insert(U(1, 1), U(4, 0), U(2, 6)))
    rows = _walks_equal(g, ex, starts)
    assert rows[1, 1] in (4, 0)
    # every out-edge of vertex 0 deleted: a dead end, tombstones stay
    g.delete_batch(U(0, 0, 0), U(2, 0, 1))
    assert ex.delete(U(0, 0, 0), U(2, 0, 1)) == 0
    d = g.dump()
    assert_exact_equal(d, ex.dump())
    assert d["live"][0] == 0 and d["ecnt"][0] == 3 and d["am"][0] == 0
    rows = _walks_equal(g, ex, starts)
    assert (rows[0, 1:] == -1).all()
    # and revives: the new edge takes slot 3
    assert list(g.insert_batch(U(0), U(5), U(1))) == [3]
    ex.insert(U(0), U(5), U(1))
    rows = _walks_equal(g, ex, starts)
    assert rows[0, 1] == 5
    check_exact_invariants(g.dump(), n)


def test_extreme_weights_and_self_loops():
    n = 6
    g, ex = _pair(n)
    src = U(0, 0, 0, 0, 1, 2, 2)
    dst = U(1, 2, 3, 0, 1, 2, 3)  # 0 -> 0, 1 -> 1, 2 -> 2 self-loops
    w = U(1, 1 << 31, 0xFFFFFFFF, 0x80000001, 0xFFFFFFFF, 3, 0x7FFFFFFF)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    assert_exact_equal(g.dump(), ex.dump())
    starts = np.repeat(np.arange(n, dtype=np.uint32), 50)
    rows = _walks_equal(g, ex, starts, length=20)
    assert (rows[50:100, 1:] == 1).all()  # vertex 1 only loops to itself
    check_exact_invariants(g.dump(), n)


def test_empty_graph_then_growth():
    n = 16
    g, ex = _pair(n)
    g.load_edges(U(), U(), U(), n)
    ex.load(U(), U(), U())
    starts = np.arange(n, dtype=np.uint32)
    rows = _walks_equal(g, ex, starts)
    assert (rows[:, 1:] == -1).all() and np.array_equal(rows[:, 0], starts)
    rng = np.random.default_rng(2)
    s, d = rng.integers(0, n, 200).astype(np.uint32), rng.integers(0, n, 200).astype(np.uint32)
    ww = rng.integers(1, 1 << 32, 200, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(g.insert_batch(s, d, ww), ex.insert(s, d, ww))
    assert_exact_equal(g.dump(), ex.dump())
    _walks_equal(g, ex, starts, length=30)
