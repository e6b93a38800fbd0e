"""The CPU oracle's sampler against the definitions it restates, with no GPU:
one-hop draws against P(v | u) = w(u, v) / sum of w(u, .)
(include/Bingo.cuh:220-267), node2vec second steps against
w(cur, x) * alpha(prev, x) (include/operation.cuh:281-335, with the
neighbour test on N(prev)), and PPR walk lengths against the geometric stop
of include/operation.cuh:336-368, and one-hop draws of 16.16 fixed-point
weights against the float weights they quantise (include/Bingo.cuh:65-69,
:254-264). Pearson's chi-square at alpha = 1e-3 per
test (Bonferroni over the vertices where several are tested). The CUDA walks
equal the oracle's bit for bit, so this pins both to the distributions."""
import numpy as np
import pytest

from bingo_b200 import gen
from oracle import pyoracle as po
from tests.helpers import chisq_pvalue

ALPHA = 1e-3
DEEPWALK, NODE2VEC, PPR, SAMPLING = 0, 1, 2, 3


def test_one_hop_every_bit_group():
    """Weights chosen so that bit groups from 0 to 31 carry mass, some with
    one member and some with several."""
    n = 64
    w0 = np.array([1, 2, 3, 1000, 65535, 2 ** 20 + 7, 2 ** 31 + 5, 12, 12, 999], np.uint64)
    ex = po.ExactGraph(n)
    ex.load(np.zeros(len(w0), np.uint32), np.arange(1, len(w0) + 1, dtype=np.uint32), w0.astype(np.uint32))
    out = ex.walk(SAMPLING, 1, np.zeros(1_000_000, np.uint32), seed=2024)
    counts = np.bincount(out, minlength=n)[1:len(w0) + 1]
    assert counts.sum() == len(out)
    pv = chisq_pvalue(counts, w0 / w0.sum())
    assert pv > ALPHA, pv


def test_one_hop_rmat_hubs_after_updates():
    """The highest-degree vertices of an R-MAT graph with log-uniform weights,
    after an insert and a delete batch (the distribution is over live edges
    only, parallel edges adding their weights)."""
    scale = 11
    n = 1 << scale
    src, dst = gen.rmat(scale, 16, seed=91)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 20, seed=92)
    ug = gen.UpdateGen(n, src, dst, seed=93)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    i_s, i_d, i_w = ug.inserts(4000, gen.W_LOGUNIFORM, 1, 2 ** 20)
    ex.insert(i_s, i_d, i_w)
    d_u, d_slot = ug.deletes(4000)
    assert ex.delete(d_u, d_slot) == 0
    # live edges of the updated graph, from the oracle's own slot dump
    st = ex.dump()
    ecnt = st["ecnt"].astype(np.int64)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(ecnt, out=off[1:])
    deg = np.asarray(st["live"], np.int64)
    tested = np.argsort(-deg)[:12]
    reps = 150_000
    out = ex.walk(SAMPLING, 1, np.repeat(tested.astype(np.uint32), reps), seed=31).reshape(len(tested), reps)
    alpha = ALPHA / len(tested)
    for i, u in enumerate(tested):
        v = st["ev"][off[u]:off[u + 1]].astype(np.int64)
        ww = st["ew"][off[u]:off[u + 1]].astype(np.float64)
        probs = np.zeros(n)
        np.add.at(probs, v[ww > 0], ww[ww > 0])
        probs /= probs.sum()
        pv = chisq_pvalue(np.bincount(out[i], minlength=n), probs)
        assert pv > alpha, (int(u), pv)


@pytest.mark.parametrize("p,q", [(0.25, 4.0), (0.5, 2.0), (4.0, 0.25), (1.0, 1.0)])
def test_node2vec_second_step(p, q):
    """From prev = 0, cur = 1: x = 0 returns (1/p), x in {2, 3} are
    out-neighbours of prev (1), x in {4, 5} are not (1/q). Covers the return
    region (1/p above max(1, 1/q)) and plain rejection."""
    n = 16
    edges = [(0, 1, 2 ** 30), (0, 2, 1), (0, 3, 1),
             (1, 0, 7), (1, 2, 3), (1, 3, 11), (1, 4, 5), (1, 5, 13)]
    ex = po.ExactGraph(n)
    ex.load(np.array([e[0] for e in edges], np.uint32), np.array([e[1] for e in edges], np.uint32),
            np.array([e[2] for e in edges], np.uint32))
    rows = ex.walk(NODE2VEC, 3, np.zeros(600_000, np.uint32), seed=17, p=p, q=q)
    rows = rows[rows[:, 1] == 1]
    alpha = {0: 1 / p, 2: 1.0, 3: 1.0, 4: 1 / q, 5: 1 / q}
    probs = np.zeros(n)
    for (u, v, wt) in edges:
        if u == 1:
            probs[v] += wt * alpha[v]
    probs /= probs.sum()
    pv = chisq_pvalue(np.bincount(rows[:, 2], minlength=n), probs)
    assert pv > ALPHA, (p, q, pv)


@pytest.mark.parametrize("stop", [0.15, 0.0125])
def test_ppr_stops_geometrically(stop):
    """On a graph with no dead end a PPR walk stops after each move with
    probability `stop`: K moves with P(K = k) = (1 - stop)^(k - 1) * stop for
    k < L - 1, and the rest of the mass at K = L - 1 (the row is full)."""
    n, L = 256, 40
    u = np.arange(n, dtype=np.uint32)
    src = np.concatenate([u, u])
    dst = np.concatenate([(u + 1) % n, (u + 7) % n]).astype(np.uint32)
    ex = po.ExactGraph(n)
    ex.load(src, dst, np.full(len(src), 3, np.uint32))
    rows = ex.walk(PPR, L, np.tile(u, 1000), seed=5, stop=stop)
    moves = (rows >= 0).sum(axis=1) - 1
    assert moves.min() >= 1 and moves.max() <= L - 1
    k = np.arange(1, L)
    probs = (1 - stop) ** (k - 1) * stop
    probs[-1] = (1 - stop) ** (L - 2)
    pv = chisq_pvalue(np.bincount(moves, minlength=L)[1:], probs)
    assert pv > ALPHA, (stop, pv)


def test_float_weights_one_hop():
    """Float-weight mode's parity definition on the oracle: weights quantised
    to 16.16 fixed point (bingo_weights_to_fixed16) and loaded as integers
    give one-hop draws that pass against the float weights themselves (the
    quantisation moves each probability by at most 2^-17 / w relative)."""
    from bingo_b200 import fixed16
    n = 64
    w = np.array([0.001, 0.37, 1.0, 2.5, 3.25, 17.125, 999.9, 12345.678, 65535.5, 0.75], np.float32)
    ex = po.ExactGraph(n)
    ex.load(np.zeros(len(w), np.uint32), np.arange(1, len(w) + 1, dtype=np.uint32), fixed16(w))
    out = ex.walk(SAMPLING, 1, np.zeros(1_000_000, np.uint32), seed=77)
    probs = w.astype(np.float64) / w.astype(np.float64).sum()
    pv = chisq_pvalue(np.bincount(out, minlength=n)[1:len(w) + 1], probs)
    assert pv > ALPHA, pv
