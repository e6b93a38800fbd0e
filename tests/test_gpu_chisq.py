"""Distribution check: per-vertex empirical transition frequencies of the
CUDA sampler against the exact weight-proportional distribution
P(v | u) = sum of w(u, v) / sum of w(u, .), by Pearson's chi-square test at
significance alpha = 1e-3 per vertex (Bonferroni over the vertices tested)."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, SAMPLING, Graph, gen
from tests.helpers import chisq_pvalue as _chisq

pytestmark = pytest.mark.gpu
ALPHA = 1e-3


def test_one_hop_distribution_handmade():
    """Weights chosen so every bit group, dense and sparse, carries mass."""
    n = 64
    w0 = np.array([1, 2, 3, 1000, 65535, 2 ** 20 + 7, 2 ** 31 + 5, 12, 12, 999], np.uint64)
    src = np.zeros(len(w0), np.uint32)
    dst = np.arange(1, len(w0) + 1, dtype=np.uint32)
    g = Graph()
    g.load_edges(src, dst, w0.astype(np.uint32), n)
    draws = 2_000_000
    out = g.walk(app=SAMPLING, starts=np.zeros(draws, np.uint32), seed=2024)
    counts = np.bincount(out, minlength=n)[1:len(w0) + 1].astype(np.float64)
    p = _chisq(counts, w0 / w0.sum())
    assert p > ALPHA, p


def test_walk_transition_distribution_rmat():
    n_scale = 12
    n = 1 << n_scale
    src, dst = gen.rmat(n_scale, 16, seed=77)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 20, seed=78)
    g = Graph()
    g.load_edges(src, dst, w, n)
    deg = np.bincount(src, minlength=n)
    test_vertices = np.argsort(-deg)[:20]
    # one-hop draws from the tested vertices, many per vertex
    reps = 200_000
    starts = np.repeat(test_vertices.astype(np.uint32), reps)
    out = g.walk(app=SAMPLING, starts=starts, seed=31).reshape(len(test_vertices), reps)
    alpha = ALPHA / len(test_vertices)
    for i, u in enumerate(test_vertices):
        sel = src == u
        probs = np.zeros(n)
        np.add.at(probs, dst[sel], w[sel].astype(np.float64))
        probs /= probs.sum()
        counts = np.bincount(out[i], minlength=n).astype(np.float64)
        pv = _chisq(counts, probs)
        assert pv > alpha, (int(u), pv)
    # multi-step walks: every transition follows an existing edge
    rows = g.walk(app=DEEPWALK, length=80, first=0, n_starts=n, seed=5)
    a, b = rows[:, :-1].ravel(), rows[:, 1:].ravel()
    ok = b >= 0
    keys = set((src.astype(np.int64) << 32 | dst).tolist())
    pairs = (a[ok].astype(np.int64) << 32) | b[ok]
    assert all(x in keys for x in np.unique(pairs).tolist())


@pytest.mark.parametrize("p,q", [(0.25, 4.0), (0.5, 2.0), (4.0, 0.25), (1.0, 1.0)])
def test_node2vec_second_order_distribution(p, q):
    """Second step of node2vec walks from a fixed (prev, cur) pair against
    P(x) ~ w(cur, x) * alpha(prev, x), alpha = 1/p (x = prev), 1 (x a
    neighbour of prev), 1/q (other). Covers the return region (1/p above the
    envelope max(1, 1/q)) and plain rejection."""
    from bingo_b200 import NODE2VEC
    n = 16
    # prev = 0 steps to cur = 1 almost surely; 0's other out-neighbours 2, 3
    # make them "in" candidates at cur.
    edges = [(0, 1, 2 ** 30), (0, 2, 1), (0, 3, 1),
             (1, 0, 7), (1, 2, 3), (1, 3, 11), (1, 4, 5), (1, 5, 13)]
    src = np.array([e[0] for e in edges], np.uint32)
    dst = np.array([e[1] for e in edges], np.uint32)
    w = np.array([e[2] for e in edges], np.uint32)
    g = Graph()
    g.load_edges(src, dst, w, n)
    rows = g.walk(app=NODE2VEC, length=3, starts=np.zeros(1_000_000, np.uint32), p=p, q=q, seed=17)
    rows = rows[rows[:, 1] == 1]
    counts = np.bincount(rows[:, 2], minlength=n).astype(np.float64)
    alpha = {0: 1 / p, 2: 1.0, 3: 1.0, 4: 1 / q, 5: 1 / q}
    probs = np.zeros(n)
    for (u, v, wt) in edges:
        if u == 1:
            probs[v] += wt * alpha[v]
    probs /= probs.sum()
    pv = _chisq(counts, probs)
    assert pv > ALPHA, (p, q, pv, counts[:6] / counts.sum(), probs[:6])
