"""Graph snapshots: a restored handle holds exactly the saved store, so it
walks and updates like the handle that saved it (checked against the
oracle), and damaged or mismatched files are refused."""
import numpy as np
import pytest

from bingo_b200 import BATCHED, DEEPWALK, NODE2VEC, PPR, SAMPLING, BingoError, Graph, WalkJob, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, workload

pytestmark = pytest.mark.gpu


def _built(node2vec=True):
    n, src, dst, w, ops = workload(scale=11, ef=12, seed=77, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 28, rounds=3,
                                   k_ins=4000, k_del=3000)
    g, ex = Graph(node2vec=node2vec), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    for op in ops[:-2]:
        if op[0] == "ins":
            g.insert_batch(*op[1:])
            ex.insert(*op[1:])
        else:
            g.delete_batch(*op[1:])
            ex.delete(*op[1:])
    return n, g, ex, ops[-2:]


def test_restore_reproduces_state_walks_and_updates(tmp_path):
    n, g, ex, tail = _built()
    path = tmp_path / "g.snap"
    g.save(path)
    h = Graph(node2vec=True)
    h.load_edges(np.array([0], np.uint32), np.array([1], np.uint32), np.array([5], np.uint32), 3)  # replaced
    h.restore(path)
    assert h.n == n
    assert_exact_equal(h.dump(), g.dump())
    assert_exact_equal(h.dump(), ex.dump())
    starts = np.arange(0, n, 3, dtype=np.uint32)
    for app, L in ((DEEPWALK, 30), (NODE2VEC, 20), (PPR, 40), (SAMPLING, 1)):
        a = h.walk(app=app, length=L, starts=starts, seed=3, job_id=app)
        assert np.array_equal(a, g.walk(app=app, length=L, starts=starts, seed=3, job_id=app))
        assert np.array_equal(a, ex.walk(app, L, starts, seed=3, job_id=app))
    ins, dele = tail
    assert np.array_equal(h.insert_batch(*ins[1:]), ex.insert(*ins[1:]))
    h.delete_batch(*dele[1:])
    ex.delete(*dele[1:])
    assert_exact_equal(h.dump(), ex.dump())


def test_snapshot_refuses_mismatch_and_damage(tmp_path):
    n, g, ex, _ = _built(node2vec=False)
    path = tmp_path / "g.snap"
    g.save(path)
    with pytest.raises(BingoError) as e:
        Graph(node2vec=True).restore(path)
    assert e.value.name == "BINGO_ERR_UNSUPPORTED"
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.snap"
    raw[len(raw) // 2] ^= 0x40
    bad.write_bytes(bytes(raw))
    h = Graph(node2vec=False)
    with pytest.raises(BingoError, match="checksum"):
        h.restore(bad)
    with pytest.raises(BingoError):  # a failed restore leaves no graph
        h.walk(app=DEEPWALK, length=5, starts=np.zeros(4, np.uint32))
    short = tmp_path / "short.snap"
    short.write_bytes(path.read_bytes()[:-100])
    with pytest.raises(BingoError, match="truncated"):
        h.restore(short)
    junk = tmp_path / "junk.snap"
    junk.write_bytes(b"not a snapshot at all" * 10)
    with pytest.raises(BingoError, match="not a graph snapshot"):
        h.restore(junk)
    h.restore(path)  # a good file still restores afterwards
    assert_exact_equal(h.dump(), ex.dump())
