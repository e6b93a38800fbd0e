"""Batched programs (bingo_run): walk-job sets and update batches in one
ordered sequence with no host synchronisation, directly or captured into a
CUDA graph. Results must equal the oracle replaying the same sequence."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING, BingoError, Graph, WalkJob, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal

pytestmark = pytest.mark.gpu


def _program(torch, n, ug, rng, seed, n_phases=3):
    """Alternating walk sets and update batches, device tensors."""
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()  # noqa: E731
    ops, host = [], []
    specs = [(DEEPWALK, 30, {}), (NODE2VEC, 20, dict(p=0.25, q=4.0)), (PPR, 60, dict(stop_prob=0.15)),
             (SAMPLING, 1, {})]
    jid = 0
    for ph in range(n_phases):
        jobs, hjobs = [], []
        for app, L, kw in specs:
            k = int(rng.integers(50, 3000))
            starts = rng.integers(0, n, size=k).astype(np.uint32)
            shape = (k,) if app == SAMPLING else (k, L)
            out = torch.full(shape, -5, dtype=torch.int32, device="cuda")
            jobs.append(WalkJob(app=app, length=L, starts=t(starts), n_starts=k, seed=seed, job_id=jid, out=out,
                                p=kw.get("p", 0.5), q=kw.get("q", 2.0), stop_prob=kw.get("stop_prob", 0.0125)))
            hjobs.append((app, L, starts, jid, kw))
            jid += 1
        ops.append(("walk", jobs))
        host.append(("walk", hjobs))
        ins = ug.inserts(int(rng.integers(100, 2000)), gen.W_UNIFORM, 1, 65535)
        slots = torch.empty(len(ins[0]), dtype=torch.int32, device="cuda")
        ops.append(("insert", t(ins[0]), t(ins[1]), t(ins[2]), slots))
        host.append(("insert",) + ins + (slots,))
        dels = ug.deletes(int(rng.integers(100, 2000)))
        ops.append(("delete", t(dels[0]), t(dels[1])))
        host.append(("delete",) + dels)
    return ops, host


def _replay_oracle(ex, host, seed, outs):
    for op, o in zip(host, outs):
        if op[0] == "walk":
            for (app, L, starts, jid, kw), job in zip(op[1], o[1]):
                ref = ex.walk(app, L, starts, seed=seed, job_id=jid, p=kw.get("p", 0.5), q=kw.get("q", 2.0),
                              stop=kw.get("stop_prob", 0.0125))
                assert np.array_equal(job.out.cpu().numpy(), ref), (app, jid)
        elif op[0] == "insert":
            slots = ex.insert(*op[1:4])
            assert np.array_equal(op[4].cpu().numpy().view(np.uint32), slots)
        else:
            assert ex.delete(*op[1:3]) == 0


@pytest.mark.parametrize("graph", [False, True])
def test_program_matches_oracle(graph):
    torch = pytest.importorskip("torch")
    n = 1 << 12
    src, dst = gen.rmat(12, 16, seed=61)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 65535, seed=62)
    g = Graph()
    g.load_edges(src, dst, w, n)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=63)
    ops, host = _program(torch, n, ug, np.random.default_rng(64), seed=123)
    g.run(ops, graph=graph)
    _replay_oracle(ex, host, 123, ops)
    assert_exact_equal(g.dump(), ex.dump())


def test_graph_replay_with_new_contents():
    """Same shape, new job seeds and new batch contents: the captured graph is
    replayed (job tables re-uploaded), and results still match the oracle."""
    torch = pytest.importorskip("torch")
    n = 1 << 12
    src, dst = gen.rmat(12, 16, seed=71)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 1024, seed=72)
    g = Graph()
    g.load_edges(src, dst, w, n)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    ug = gen.UpdateGen(n, src, dst, seed=73)
    rng = np.random.default_rng(74)
    ops, host = _program(torch, n, ug, rng, seed=5, n_phases=2)
    g.run(ops, graph=True)
    _replay_oracle(ex, host, 5, ops)
    launches = g.stats()["kernel_launches"]
    # refill the same device buffers with the next batches, change the seeds
    for idx, op in enumerate(ops):
        if op[0] == "insert":
            k = op[1].numel()
            ins = ug.inserts(k, gen.W_UNIFORM, 1, 1024)
            for dev, col in zip(op[1:4], ins):
                dev.copy_(torch.from_numpy(col.view(np.int32)))
            host[idx] = ("insert",) + ins + (op[4],)
        elif op[0] == "delete":
            k = op[1].numel()
            dels = ug.deletes(k)
            assert len(dels[0]) == k
            for dev, col in zip(op[1:3], dels):
                dev.copy_(torch.from_numpy(col.view(np.int32)))
            host[idx] = ("delete",) + dels
        else:
            for j in op[1]:
                j.seed = 6
    g.run(ops, graph=True)
    _replay_oracle(ex, host, 6, ops)
    assert_exact_equal(g.dump(), ex.dump())
    assert g.stats()["kernel_launches"] > launches


def test_program_rejects_host_arrays():
    torch = pytest.importorskip("torch")
    n = 1 << 8
    src, dst = gen.rmat(8, 8, seed=75)
    g = Graph()
    g.load_edges(src, dst, gen.weights(len(src), seed=76), n)
    with pytest.raises(BingoError) as e:
        g.run([("insert", np.array([1], np.uint32), np.array([2], np.uint32), np.array([3], np.uint32))])
    assert e.value.name == "BINGO_ERR_INVALID_ARGUMENT"
