"""Tuning knobs and the autotuner: no knob changes any walk, slot id or graph
state (checked against the oracle), and autotuning leaves the graph as it
found it."""
import numpy as np
import pytest

from bingo_b200 import BATCHED, DEEPWALK, NODE2VEC, PPR, BingoError, Graph, WalkJob, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, workload

pytestmark = pytest.mark.gpu


def _jobs(n, rng, torch):
    out = []
    for j, (app, L, k) in enumerate([(DEEPWALK, 40, 3000), (NODE2VEC, 25, 2000), (PPR, 60, 2500),
                                     (DEEPWALK, 7, 500)]):
        st = rng.integers(0, n, size=k).astype(np.uint32)
        out.append(WalkJob(app=app, length=L, starts=torch.from_numpy(st.view(np.int32)).cuda(), n_starts=k,
                           job_id=j, seed=11, stop_prob=0.15,
                           out=torch.empty((k, L), dtype=torch.int32, device="cuda")))
    return out


def _oracle_rows(ex, jobs):
    return [ex.walk(j.app, j.length, j.starts.cpu().numpy().view(np.uint32), seed=j.seed, job_id=j.job_id,
                    stop=j.stop_prob) for j in jobs]


@pytest.mark.parametrize("knobs", [dict(walk_chunk=1), dict(walk_chunk=256, walk_order=0),
                                   dict(walk_split=1, walk_blocks_per_sm=2), dict(walk_chunk=7, walk_blocks_per_sm=1)])
def test_walk_knobs_do_not_change_walks(knobs):
    import torch
    n, src, dst, w, _ = workload(scale=11, ef=8, seed=5, rounds=0)
    g, ex = Graph(), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    g.set_tuning(**knobs)
    assert all(g.tuning()[k] == v for k, v in knobs.items())
    jobs = _jobs(n, np.random.default_rng(3), torch)
    g.walk_jobs(jobs, mode=BATCHED)
    for j, ref in zip(jobs, _oracle_rows(ex, jobs)):
        assert np.array_equal(j.out.cpu().numpy(), ref)


@pytest.mark.parametrize("chunk,apply_bps", [(1000, 8), (4096, 1), (1, 32)])
def test_update_chunks_give_identical_state(chunk, apply_bps):
    n, src, dst, w, ops = workload(scale=10, ef=16, seed=29, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 30, rounds=3,
                                   k_ins=9000, k_del=7000)
    g, ex = Graph(), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    g.set_tuning(update_chunk=chunk, apply_blocks_per_sm=apply_bps)
    for op in ops:
        if op[0] == "ins":
            assert np.array_equal(g.insert_batch(*op[1:]), ex.insert(*op[1:]))
        else:
            g.delete_batch(*op[1:])
            ex.delete(*op[1:])
    assert_exact_equal(g.dump(), ex.dump())


def test_chunked_batches_keep_all_or_nothing_and_skip_counts():
    import torch
    n, src, dst, w, ops = workload(scale=9, ef=8, seed=31, rounds=1, k_ins=3000, k_del=3000)
    g = Graph()
    g.load_edges(src, dst, w, n)
    g.set_tuning(update_chunk=500)
    before = g.dump()
    s, d, ww = (torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda() for x in ops[0][1:4])
    ww[2900] = 0  # a zero weight in the last sub-batch rejects the whole batch
    with pytest.raises(BingoError) as e:
        g.insert_batch(s, d, ww, return_slots=False)
    assert e.value.name == "BINGO_ERR_ZERO_WEIGHT"
    assert_exact_equal(g.dump(), before)
    g.insert_batch(*ops[0][1:4], return_slots=False)
    # Deletes: absent slots in several sub-batches are all skipped and counted.
    u, sl = ops[1][1], ops[1][2].copy()
    sl[[10, 1200, 2500]] = 10 ** 6
    with pytest.raises(BingoError) as e:
        g.delete_batch(u, sl)
    assert "3 deletes of absent slots" in str(e.value)


def test_autotune_leaves_graph_unchanged_and_picks_valid_knobs():
    import torch
    n, src, dst, w, ops = workload(scale=12, ef=16, seed=41, rounds=1, k_ins=40000, k_del=40000)
    g = Graph()
    g.load_edges(src, dst, w, n)
    before = g.dump()
    jobs = _jobs(n, np.random.default_rng(9), torch)
    rep = g.autotune(jobs, inserts=ops[0][1:4], deletes=ops[1][1:3], repeats=2)
    assert rep["candidates"] >= 8
    assert rep["walk_ms_best"] <= rep["walk_ms_start"] and rep["update_ms_best"] <= rep["update_ms_start"]
    assert g.tuning() == rep["best"]
    assert_exact_equal(g.dump(), before)
    # The tuned handle still computes the same walks and updates as the oracle.
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    g.walk_jobs(jobs, mode=BATCHED)
    for j, ref in zip(jobs, _oracle_rows(ex, jobs)):
        assert np.array_equal(j.out.cpu().numpy(), ref)
    assert np.array_equal(g.insert_batch(*ops[0][1:4]), ex.insert(*ops[0][1:4]))
    g.delete_batch(*ops[1][1:3])
    ex.delete(*ops[1][1:3])
    assert_exact_equal(g.dump(), ex.dump())


def test_invalid_tuning_rejected():
    n, src, dst, w, _ = workload(scale=8, ef=4, seed=2, rounds=0)
    g = Graph()
    g.load_edges(src, dst, w, n)
    for bad in (dict(walk_chunk=1025), dict(walk_chunk=2048), dict(apply_blocks_per_sm=0), dict(walk_split=2)):
        with pytest.raises(BingoError):
            g.set_tuning(**bad)
    with pytest.raises(ValueError):
        g.set_tuning(nonsense=1)


def test_autotune_cache_reuses_knobs(tmp_path):
    import json

    import torch
    n, src, dst, w, ops = workload(scale=11, ef=16, seed=43, rounds=1, k_ins=20000, k_del=20000)
    cache = str(tmp_path / "tuning.json")
    g = Graph()
    g.load_edges(src, dst, w, n)
    jobs = _jobs(n, np.random.default_rng(12), torch)
    first = g.autotune(jobs, inserts=ops[0][1:4], deletes=ops[1][1:3], repeats=1, cache=cache)
    assert not first["cached"] and first["candidates"] > 0
    table = json.load(open(cache))
    assert len(table) == 1 and list(table.values())[0] == first["best"]
    h = Graph()  # a new handle on the same GPU and workload shape takes the stored knobs
    h.load_edges(src, dst, w, n)
    h.set_tuning(walk_chunk=128)
    again = h.autotune(jobs, inserts=ops[0][1:4], deletes=ops[1][1:3], repeats=1, cache=cache)
    assert again["cached"] and again["candidates"] == 0 and h.tuning() == first["best"]
