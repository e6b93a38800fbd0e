"""Delete by (u, v) pair through the C ABI against the oracle: the r-th
repeat of a pair deletes the r-th lowest live slot of u with neighbour v,
absent pairs are skipped and reported, and the resulting graph state is
bit-exact."""
import numpy as np
import pytest

from bingo_b200 import NODE2VEC, BingoError, Graph, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, check_exact_invariants

pytestmark = pytest.mark.gpu


def _graph_with_parallel_edges(scale, seed):
    n = 1 << scale
    src, dst = gen.rmat(scale, 8, seed=seed)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 24, seed=seed + 1)
    rng = np.random.default_rng(seed)
    # Parallel edges: re-insert existing pairs up to three times.
    pick = rng.choice(len(src), size=len(src) // 4)
    reps = rng.integers(1, 4, size=len(pick))
    ps = np.repeat(src[pick], reps).astype(np.uint32)
    pd = np.repeat(dst[pick], reps).astype(np.uint32)
    pw = rng.integers(1, 1 << 20, size=len(ps)).astype(np.uint32)
    return n, src, dst, w, (ps, pd, pw)


@pytest.mark.parametrize("scale,seed", [(8, 3), (12, 41)])
def test_delete_pairs_matches_oracle(scale, seed):
    n, src, dst, w, par = _graph_with_parallel_edges(scale, seed)
    g, ex = Graph(node2vec=True), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    g.insert_batch(*par)
    ex.insert(*par)
    rng = np.random.default_rng(seed + 7)
    for rnd in range(3):
        live_u, live_v = par[0], par[1]
        k = len(src) // 3
        i = rng.choice(len(src), size=k)
        u = np.concatenate([src[i], live_u[: k // 4], rng.integers(0, n, size=k // 8)]).astype(np.uint32)
        v = np.concatenate([dst[i], live_v[: k // 4], rng.integers(0, n, size=k // 8)]).astype(np.uint32)
        perm = rng.permutation(len(u))
        u, v = u[perm], v[perm]
        bad, _ = ex.delete_pairs(u, v)
        assert bad > 0  # repeats beyond the live multiplicity and random absent pairs
        with pytest.raises(BingoError) as e:
            g.delete_pairs(u, v)
        assert "absent" in str(e.value)
        assert_exact_equal(g.dump(), ex.dump(), f"round {rnd}: ")
    check_exact_invariants(g.dump(), n)
    # Walks on the result agree as well (second-order adjacency included).
    starts = np.arange(min(n, 2048), dtype=np.uint32)
    assert np.array_equal(g.walk(app=NODE2VEC, length=20, starts=starts, seed=5),
                          ex.walk(NODE2VEC, 20, starts, seed=5))


def test_delete_pairs_all_present_is_ok():
    n, src, dst, w, _ = _graph_with_parallel_edges(9, 5)
    g, ex = Graph(node2vec=False), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    sel = np.random.default_rng(1).choice(len(src), size=len(src) // 2, replace=False)
    g.delete_pairs(src[sel], dst[sel])
    bad, slots = ex.delete_pairs(src[sel], dst[sel])
    assert bad == 0
    assert_exact_equal(g.dump(), ex.dump())


def test_delete_pairs_out_of_range_rejects_batch():
    n, src, dst, w, _ = _graph_with_parallel_edges(8, 9)
    g, ex = Graph(), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    before = g.dump()
    u = np.array([src[0], src[1]], np.uint32)
    v = np.array([dst[0], n + 5], np.uint32)
    import torch
    with pytest.raises(BingoError):
        g.delete_pairs(torch.from_numpy(u.view(np.int32)).cuda(), torch.from_numpy(v.view(np.int32)).cuda())
    assert_exact_equal(g.dump(), before)


def test_delete_pairs_in_programs_and_serving():
    """The same translation inside a captured program (replayed with new
    contents) and as a served update: state equals the oracle's."""
    import torch
    n, src, dst, w, par = _graph_with_parallel_edges(10, 13)
    rng = np.random.default_rng(4)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()  # noqa: E731
    g, ex = Graph(node2vec=True), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    k = 3000
    for rnd in range(2):  # second round replays the captured graph with new batch contents
        i = rng.choice(len(src), size=k)
        u = np.concatenate([src[i], par[0][:500]]).astype(np.uint32)
        v = np.concatenate([dst[i], par[1][:500]]).astype(np.uint32)
        if rnd == 0:
            du, dv = dev(u), dev(v)
        else:
            du.copy_(dev(u))
            dv.copy_(dev(v))
        bad, _ = ex.delete_pairs(u, v)
        if bad:  # repeats beyond a pair's live edges: skipped, reported after the rest applied
            with pytest.raises(BingoError, match="absent"):
                g.run([("delete_pairs", du, dv)], graph=True)
        else:
            g.run([("delete_pairs", du, dv)], graph=True)
        assert_exact_equal(g.dump(), ex.dump(), f"program round {rnd}: ")
    g.serve_start(output_budget_bytes=64 << 20, max_update_batch=1000)  # chunks see earlier chunks' deletes
    i = rng.choice(len(src), size=k)
    u, v = src[i].astype(np.uint32), dst[i].astype(np.uint32)
    t, _ = g.submit_update("delete_pairs", u, v)
    st = g.serve_wait(t)
    g.serve_stop()
    bad, _ = ex.delete_pairs(u, v)
    assert st["done"] and (st["status"] == 0) == (bad == 0)
    assert_exact_equal(g.dump(), ex.dump(), "served: ")
