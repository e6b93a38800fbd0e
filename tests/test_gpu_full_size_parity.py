"""Bit-exact parity at the full size of the DeepWalk, node2vec and batched
workloads, against the CPU oracle (ExactGraph) fed the same inputs.

DeepWalk workload: R-MAT scale 20 (16.1 M edges), log-uniform weights in
[1, 2^20), the bench's own generator and batches. After the load and after
each of two 50K + 50K update batches the whole store (every slot, group
member list in order, back-pointer, alias slot) equals the oracle's and the
insert slot ids equal the oracle's; then all 1,048,576 walks of length 80 are
compared row for row (the state and walk semantics of include/operation.cuh:
122-214 and :252-280, restated exactly).

node2vec workload: R-MAT scale 22 (65 M edges), Zipf(1.2) weights on
[1, 2^24), one 500K + 500K batch, the whole store compared after the load
and after the batch, then a 65,536-walk sample of node2vec (p = 0.5, q = 2)
walks of length 40 compared row for row (include/operation.cuh:281-335)."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PLAIN, Graph, WalkJob
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal

pytestmark = pytest.mark.gpu


def _compare_state(g, ex, what):
    a = g.dump()
    b = ex.dump()
    assert_exact_equal(a, b, what)
    del a, b


def test_deepwalk_rmat20_state_after_every_batch_and_all_walks():
    import torch

    import bench
    n, src, dst, w, batches = bench.make_workload(2)
    g = Graph(node2vec=False)
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    _compare_state(g, ex, "load: ")
    for i, (ins, dels) in enumerate(batches):
        slots = g.insert_batch(*ins)
        assert np.array_equal(slots, ex.insert(*ins)), f"batch {i}: insert slot ids"
        g.delete_batch(*dels)
        assert ex.delete(*dels) == 0
        _compare_state(g, ex, f"batch {i}: ")
    seed, job = 0xB1460, 5
    out = torch.empty((n, bench.WALK_LEN), dtype=torch.int32, device="cuda")
    g.walk_jobs([WalkJob(app=DEEPWALK, length=bench.WALK_LEN, n_starts=n, first=0, job_id=job, seed=seed, out=out)],
                mode=PLAIN)
    g.sync()
    rows = out.cpu().numpy()
    ref = ex.walk_interleaved(DEEPWALK, bench.WALK_LEN, np.arange(n, dtype=np.uint32), seed=seed, job_id=job)
    bad = np.nonzero((rows != ref).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of {n} walks differ, first {bad[:5]}"
    assert (rows[:, 1:] >= 0).sum() > 0  # (R-MAT leaves many vertices without out-edges: their rows are -1)
    g.close()


def test_node2vec_rmat22_state_after_batch_and_walk_sample():
    import torch

    import bench
    n, src, dst, w, batches = bench.make_node2vec_workload(1)
    g = Graph(node2vec=True)
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    _compare_state(g, ex, "load: ")
    ins, dels = batches[0]
    slots = g.insert_batch(*ins)
    assert np.array_equal(slots, ex.insert(*ins)), "insert slot ids"
    g.delete_batch(*dels)
    assert ex.delete(*dels) == 0
    _compare_state(g, ex, "batch: ")
    rng = np.random.default_rng(4242)
    starts = np.sort(rng.choice(n, size=65_536, replace=False)).astype(np.uint32)
    seed, job, L = 77, 3, bench.N_LEN
    out = torch.empty((len(starts), L), dtype=torch.int32, device="cuda")
    dst_starts = torch.from_numpy(starts.view(np.int32)).cuda()
    g.walk_jobs([WalkJob(app=NODE2VEC, length=L, starts=dst_starts, n_starts=len(starts), job_id=job, seed=seed,
                         p=0.5, q=2.0, out=out)], mode=PLAIN)
    g.sync()
    rows = out.cpu().numpy()
    ref = ex.walk(NODE2VEC, L, starts, seed=seed, job_id=job, p=0.5, q=2.0)
    bad = np.nonzero((rows != ref).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of {len(starts)} walks differ, first {bad[:5]}"
    g.close()


def test_batched_program_rmat22_phase():
    """Batched workload at full size: R-MAT scale 22 (65 M edges), uniform
    [1, 65535] weights, the first phase's 16 mixed jobs (DeepWalk, node2vec
    with p, q in {0.25, 1, 4}, PPR stop 0.15; start sets of 1K-1M, lengths
    5-200) and its update chunk, run as one captured program (walks, insert,
    delete). The first 4,096 rows of every job equal the oracle's on the
    graph before the chunk, the chunk's slot ids equal the oracle's, and the
    whole store after it equals the oracle's."""
    import torch

    import bench
    from bingo_b200 import WalkJob as WJ
    n, src, dst, w, jobs, chunk, steps = bench.make_batched_workload(1)
    g = Graph(node2vec=True)
    ex = po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    phase = jobs[:bench.B_JOBS_PER_PHASE]
    ins, dels = steps[0][0]
    starts = [dev(J["starts"]) for J in phase]
    outs = [torch.empty((len(J["starts"]), J["length"]), dtype=torch.int32, device="cuda") for J in phase]
    slots = torch.empty(len(ins[0]), dtype=torch.int32, device="cuda")
    seed = 77
    walk_jobs = [WJ(app=J["app"], length=J["length"], starts=starts[k], n_starts=len(J["starts"]), job_id=J["job_id"],
                    seed=seed, p=J["p"], q=J["q"], stop_prob=J["stop_prob"], out=outs[k]) for k, J in enumerate(phase)]
    g.run([("walk", walk_jobs), ("insert", dev(ins[0]), dev(ins[1]), dev(ins[2]), slots),
           ("delete", dev(dels[0]), dev(dels[1]))], graph=True)
    g.sync()
    K = 4096
    for k, J in enumerate(phase):
        st = np.ascontiguousarray(J["starts"][:K], dtype=np.uint32)
        ref = ex.walk(J["app"], J["length"], st, seed=seed, job_id=J["job_id"], p=J["p"], q=J["q"],
                      stop=J["stop_prob"])
        got = outs[k][:len(st)].cpu().numpy()
        bad = np.nonzero((got != ref).any(axis=1))[0]
        assert len(bad) == 0, f"job {J['job_id']} (app {J['app']}, p {J['p']}, q {J['q']}): rows {bad[:5]} differ"
    assert np.array_equal(slots.cpu().numpy().view(np.uint32), ex.insert(*ins)), "chunk slot ids"
    assert ex.delete(*dels) == 0
    _compare_state(g, ex, "after the chunk: ")
    g.close()
