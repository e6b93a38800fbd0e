"""Properties at the full size of the DeepWalk workload (R-MAT scale 20,
16.1 M edges, log-uniform weights in [1, 2^20), 50K + 50K update batches,
one walk of length 80 per vertex), where a full CPU-oracle replay would take
minutes: counts add up, the device store check is clean with totals equal
to the live edge set, an insert followed by the delete of exactly its
slots restores every group count, live degree and alias mass, every walk
transition is a live edge, walks repeat exactly, and the batched launch
equals the plain one."""
import numpy as np
import pytest

from bingo_b200 import BATCHED, DEEPWALK, PLAIN, Graph, WalkJob, gen

pytestmark = pytest.mark.gpu

SCALE, EF, W_HI = 20, 16, 1 << 20


@pytest.fixture(scope="module")
def big():
    n = 1 << SCALE
    src, dst = gen.rmat(SCALE, EF, seed=1236)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, W_HI, seed=1237)
    g = Graph(node2vec=False)
    g.load_edges(src, dst, w, n)
    yield n, src, dst, w, g
    g.close()


def _group_mass(d, n):
    g = d["gcnt"].astype(np.uint64).reshape(n, 32)
    return g, (g * (np.uint64(1) << np.arange(32, dtype=np.uint64))).sum(1)


def _check_totals(g, live_weights):
    """The device store check is clean and its totals match the live edge set."""
    rep = g.check()
    assert rep["bad_vertices"] == 0 and rep["kinds"] == 0
    lw = live_weights.astype(np.uint64)
    assert rep["live_edges"] == len(lw)
    assert rep["weight_sum"] == int(lw.sum())
    assert rep["members"] == int(np.unpackbits(lw.astype(np.uint32).view(np.uint8)).sum())
    return rep


def test_counts_and_round_trip(big):
    n, src, dst, w, g = big
    st = g.stats()
    assert st["slots"] == len(src) and st["live_edges"] == len(src)
    before = g.dump()
    gc0, mass0 = _group_mass(before, n)
    assert (before["aT"].astype(np.uint64)[np.cumsum(np.r_[0, before["am"][:-1]])[before["am"] > 0]]
            == mass0[before["am"] > 0]).all()
    ug = gen.UpdateGen(n, src, dst, seed=1238)
    s, d, ww = ug.inserts(50_000, gen.W_LOGUNIFORM, 1, W_HI)
    slots = g.insert_batch(s, d, ww)
    st = g.stats()
    assert st["slots"] == len(src) + 50_000 and st["live_edges"] == len(src) + 50_000
    _check_totals(g, np.concatenate([w, ww]))
    g.delete_batch(s, slots)  # the same edges again: a full round trip
    after = g.dump()
    st = g.stats()
    assert st["live_edges"] == len(src) and st["slots"] == len(src) + 50_000  # tombstones stay
    gc1, mass1 = _group_mass(after, n)
    assert np.array_equal(gc0, gc1)
    assert np.array_equal(before["live"], after["live"])
    assert np.array_equal(before["am"], after["am"])
    # every old slot keeps its neighbour and weight; the new slots are tombstones
    ecnt0, ecnt1 = before["ecnt"].astype(np.int64), after["ecnt"].astype(np.int64)
    vert = np.repeat(np.arange(n), ecnt1)
    local = np.arange(len(after["ew"])) - np.repeat(np.cumsum(np.r_[0, ecnt1])[:-1], ecnt1)
    old = local < ecnt0[vert]
    assert np.array_equal(after["ev"][old], before["ev"]) and np.array_equal(after["ew"][old], before["ew"])
    assert (~old).sum() == 50_000 and (after["ew"][~old] == 0).all()
    rep = _check_totals(g, w)
    assert rep["alias_slots"] == int(after["am"].sum())


def test_walk_transitions_live_and_repeatable(big):
    import torch
    n, src, dst, w, g = big
    out1 = torch.empty((n, 80), dtype=torch.int32, device="cuda")
    out2 = torch.empty_like(out1)
    job = lambda o: WalkJob(app=DEEPWALK, length=80, n_starts=n, first=0, seed=99, job_id=3, out=o)  # noqa: E731
    g.walk_jobs([job(out1)], mode=PLAIN)
    g.walk_jobs([job(out2)], mode=BATCHED)
    assert torch.equal(out1, out2)
    g.walk_jobs([job(out2)], mode=PLAIN)
    assert torch.equal(out1, out2)
    rows = out1.cpu().numpy()
    steps_all = int((rows[:, 1:] >= 0).sum())
    rows = rows[::8]  # every 8th walk for the host-side edge lookups
    a, b = rows[:, :-1].ravel(), rows[:, 1:].ravel()
    ok = b >= 0
    keys = np.unique((src.astype(np.uint64) << np.uint64(32)) | dst.astype(np.uint64))
    pairs = (a[ok].astype(np.uint64) << np.uint64(32)) | b[ok].astype(np.uint64)
    idx = np.searchsorted(keys, pairs)
    assert (idx < len(keys)).all() and (keys[np.minimum(idx, len(keys) - 1)] == pairs).all()
    # -1 only after a dead end, and then to the end of the row
    dead = rows < 0
    assert (np.diff(dead.astype(np.int8), axis=1) >= 0).all()
    assert g.stats()["walk_steps"] >= 3 * steps_all
