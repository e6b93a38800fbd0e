"""Update batches at the sizes where the grouping path changes: one edge, the
8-CTA cluster's limit (12,288) and one past it (16-CTA cluster), the 16-CTA
cluster's limit (98,304) and one past it (the CUB radix-sort path), plus
vertex counts that need three 10-bit passes. The whole store and the slot
ids must equal the oracle's after every batch; batches the device rejects
change nothing."""
import numpy as np
import pytest

from bingo_b200 import BingoError, Graph, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal

pytestmark = pytest.mark.gpu


def _check_batches(n, src, dst, w, sizes, seed):
    g = Graph(node2vec=True)
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=seed)
    for k in sizes:
        ins = ug.inserts(k, gen.W_LOGUNIFORM, 1, 2 ** 20, 1.2)
        assert np.array_equal(g.insert_batch(*ins), ex.insert(*ins)), f"insert of {k}: slot ids"
        assert_exact_equal(g.dump(), ex.dump(), f"after inserting {k}: ")
        dels = ug.deletes(k)
        g.delete_batch(*dels)
        assert ex.delete(*dels) == 0
        assert_exact_equal(g.dump(), ex.dump(), f"after deleting {k}: ")
    g.close()


def test_batch_sizes_around_the_cluster_limits():
    scale = 12
    n = 1 << scale
    src, dst = gen.rmat(scale, 16, seed=501)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 20, 1.2, seed=502)
    _check_batches(n, src, dst, w, [1, 2, 1023, 12288, 12289, 65536, 98304, 98305], seed=503)


@pytest.mark.parametrize("n", [1 << 21, 3_000_000])
def test_three_digit_passes(n):
    """2^21 vertices (digits of 10, 10 and 1 bits) and 3,000,000 (10, 10, 2)."""
    rng = np.random.default_rng(504)
    m = 400_000
    src = rng.integers(0, n, size=m, dtype=np.uint32)
    dst = rng.integers(0, n, size=m, dtype=np.uint32)
    src[:2000] = n - 1  # a hub at the top of the id range
    keep = src != dst
    src, dst = src[keep], dst[keep]
    pairs = np.unique((src.astype(np.uint64) << 32) | dst)
    src, dst = (pairs >> 32).astype(np.uint32), (pairs & 0xFFFFFFFF).astype(np.uint32)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 65535, 1.2, seed=505)
    _check_batches(n, src, dst, w, [5000, 50000], seed=506)


@pytest.mark.parametrize("k", [5000, 50000])
def test_rejected_batches_on_the_cluster_path(k):
    """Device-resident batches (validated by the grouping kernel itself): an
    id >= n or a zero weight anywhere rejects the whole batch; the next valid
    batch applies normally."""
    torch = pytest.importorskip("torch")
    scale = 12
    n = 1 << scale
    src, dst = gen.rmat(scale, 16, seed=507)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 1024, 1.2, seed=508)
    g = Graph()
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=509)
    before = g.dump()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()  # noqa: E731
    a, b, c = ug.inserts(k, gen.W_UNIFORM, 1, 1024, 1.2)
    bad_dst = b.copy()
    bad_dst[k // 2] = n + 7
    with pytest.raises(BingoError) as e:
        g.insert_batch(dev(a), dev(bad_dst), dev(c), out_slots=torch.empty(k, dtype=torch.int32, device="cuda"))
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    bad_w = c.copy()
    bad_w[k - 1] = 0
    with pytest.raises(BingoError) as e:
        g.insert_batch(dev(a), dev(b), dev(bad_w), out_slots=torch.empty(k, dtype=torch.int32, device="cuda"))
    assert e.value.name == "BINGO_ERR_ZERO_WEIGHT"
    assert_exact_equal(g.dump(), before, "after rejected inserts: ")
    slots = torch.empty(k, dtype=torch.int32, device="cuda")
    g.insert_batch(dev(a), dev(b), dev(c), out_slots=slots)
    assert np.array_equal(slots.cpu().numpy().view(np.uint32), ex.insert(a, b, c))
    u, s = ug.deletes(k)
    bad_u = u.copy()
    bad_u[0] = n
    with pytest.raises(BingoError) as e:
        g.delete_batch(dev(bad_u), dev(s))
    assert e.value.name == "BINGO_ERR_OUT_OF_RANGE"
    assert_exact_equal(g.dump(), ex.dump(), "after a rejected delete: ")
    g.delete_batch(dev(u), dev(s))
    assert ex.delete(u, s) == 0
    assert_exact_equal(g.dump(), ex.dump(), "after the valid delete: ")
    g.close()
