"""Randomised operation sequences against the oracle, bit for bit. Each case
draws a small multigraph (self-loops and repeated pairs kept, vertices
without out-edges), weights from one of several bit ranges (all ones, small,
log-uniform over all 32 bits, the top bit set), and a sequence of insert
batches (new vertices' first edges included), slot deletes (absent, repeated
and tombstoned slots mixed in), deletes by pair (absent pairs mixed in) and
walks of every app with random p, q and stop probability from random start
vertices. After every operation the graph state and the walks equal the
oracle's and the device store check is clean."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING, BingoError, Graph
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal

pytestmark = pytest.mark.gpu

CASES = 24


def _weights(rng, k, kind):
    if kind == 0:
        return np.ones(k, np.uint32)
    if kind == 1:
        return rng.integers(1, 16, k).astype(np.uint32)
    if kind == 2:
        bits = rng.integers(1, 33, k)
        return np.maximum(1, (rng.random(k) * (2.0 ** bits)).astype(np.uint64)).astype(np.uint32)
    return (rng.integers(0, 2 ** 31, k).astype(np.uint64) | (1 << 31)).astype(np.uint32)


def _edges(rng, n, k):
    # a skewed source distribution leaves some vertices without out-edges
    src = np.minimum(n - 1, (rng.random(k) ** 2 * n).astype(np.uint32))
    dst = rng.integers(0, n, k).astype(np.uint32)
    return src, dst


def _live_slots(d):
    us = np.repeat(np.arange(len(d["ecnt"]), dtype=np.uint32), d["ecnt"])
    local = np.arange(len(d["ew"])) - np.repeat(np.cumsum(np.r_[0, d["ecnt"]])[:-1], d["ecnt"])
    return us, local.astype(np.uint32), d["ev"], d["ew"] != 0


@pytest.mark.parametrize("case", range(CASES))
def test_random_sequences(case):
    rng = np.random.default_rng(1000 + case)
    n = int(rng.integers(1, 400))
    kind = case % 4
    node2vec = case % 3 != 2
    m = int(rng.integers(0, 6 * n + 1))
    src, dst = _edges(rng, n, m)
    w = _weights(rng, m, kind)
    g, ex = Graph(node2vec=node2vec), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    apps = [DEEPWALK, PPR, SAMPLING] + ([NODE2VEC] if node2vec else [])
    for step in range(int(rng.integers(4, 10))):
        op = rng.integers(0, 4)
        if op == 0:  # insert
            k = int(rng.integers(1, 3 * n + 2))
            s, d = _edges(rng, n, k)
            if rng.random() < 0.5:
                s[: max(1, k // 4)] = rng.integers(0, n, max(1, k // 4))  # first edges of edgeless vertices
            ww = _weights(rng, k, int(rng.integers(0, 4)))
            assert np.array_equal(g.insert_batch(s, d, ww), ex.insert(s, d, ww))
        elif op == 1:  # delete by slot, with absent and repeated slots
            us, local, _, live = _live_slots(ex.dump())
            pick = np.flatnonzero(live)
            if len(pick) == 0:
                continue
            pick = rng.choice(pick, size=min(len(pick), int(rng.integers(1, 2 * n + 2))), replace=False)
            u, sl = us[pick], local[pick]
            extra = int(rng.integers(0, 4))
            if extra:
                u = np.concatenate([u, u[:extra], rng.integers(0, n, extra).astype(np.uint32)])
                sl = np.concatenate([sl, sl[:extra], rng.integers(0, 10 ** 6, extra).astype(np.uint32)])
            skipped = ex.delete(u, sl)
            if skipped:
                with pytest.raises(BingoError) as e:
                    g.delete_batch(u, sl)
                assert e.value.name == "BINGO_ERR_INVALID_SLOT"
            else:
                g.delete_batch(u, sl)
        elif op == 2:  # delete by pair, with absent pairs
            us, _, ev, live = _live_slots(ex.dump())
            pick = np.flatnonzero(live)
            k = int(rng.integers(1, n + 2))
            u = rng.integers(0, n, k).astype(np.uint32)
            v = rng.integers(0, n, k).astype(np.uint32)
            if len(pick):
                take = rng.choice(pick, size=min(len(pick), k), replace=True)
                u[: len(take)], v[: len(take)] = us[take], ev[take]
            skipped, _ = ex.delete_pairs(u, v)
            if skipped:
                with pytest.raises(BingoError) as e:
                    g.delete_pairs(u, v)
                assert e.value.name == "BINGO_ERR_INVALID_SLOT"
            else:
                g.delete_pairs(u, v)
        else:  # walks
            starts = rng.integers(0, n, int(rng.integers(1, 2 * n + 2))).astype(np.uint32)
            L = int(rng.integers(1, 40))
            p, q = float(rng.choice([0.25, 0.5, 1.0, 2.0, 4.0])), float(rng.choice([0.25, 0.5, 1.0, 2.0, 4.0]))
            stop = float(rng.choice([0.0125, 0.15, 0.5]))
            for app in apps:
                seed, job = int(rng.integers(0, 2 ** 31)), int(rng.integers(0, 1000))
                a = g.walk(app=app, length=L, starts=starts, seed=seed, job_id=job, p=p, q=q, stop_prob=stop)
                b = ex.walk(app, L, starts, seed=seed, job_id=job, p=p, q=q, stop=stop)
                assert np.array_equal(a, b), (case, step, app)
        assert_exact_equal(g.dump(), ex.dump(), f"case {case} step {step}")
        rep = g.check()
        assert rep["bad_vertices"] == 0
        assert rep["live_edges"] == int(ex.dump()["live"].sum())
