"""Float-weight mode (the reference's wtype::Float): weights are quantised
to 16.16 fixed point on the device, so graph state and walks are bit-exact
against the oracle fed the same fixed-point weights, and one-hop draws pass
the chi-square test against the float weights themselves (the quantisation
moves each probability by at most 2^-17 / w relative, far below what
2,000,000 draws resolve)."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, NODE2VEC, PPR, SAMPLING, BingoError, Graph, fixed16, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, chisq_pvalue as _chisq
from tests.test_gpu_chisq import ALPHA

pytestmark = pytest.mark.gpu


def _float_weights(m, seed):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(1e-3), np.log(65000.0), size=m)).astype(np.float32)


def test_float_graph_matches_oracle_on_fixed_point():
    import torch
    scale = 11
    n = 1 << scale
    src, dst = gen.rmat(scale, 12, seed=81)
    w = _float_weights(len(src), 1)
    g, ex = Graph(float_weights=True), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, fixed16(w))
    assert g.stats()["weight_mode"] == 1
    assert_exact_equal(g.dump(), ex.dump())
    ug = gen.UpdateGen(n, src, dst, seed=82)
    for r in range(3):
        s, d, _ = ug.inserts(3000, gen.W_UNIFORM, 1, 2)
        wf = _float_weights(len(s), 10 + r)
        if r == 1:  # device-resident float weights
            wf_dev = torch.from_numpy(wf).cuda()
            slots = g.insert_batch(s, d, wf_dev)
        else:
            slots = g.insert_batch(s, d, wf)
        assert np.array_equal(slots, ex.insert(s, d, fixed16(wf)))
        du, ds = ug.deletes(2000)
        g.delete_batch(du, ds)
        ex.delete(du, ds)
        assert_exact_equal(g.dump(), ex.dump(), f"round {r}: ")
    starts = np.arange(0, n, 2, dtype=np.uint32)
    for app, L in ((DEEPWALK, 40), (NODE2VEC, 25), (PPR, 40), (SAMPLING, 1)):
        assert np.array_equal(g.walk(app=app, length=L, starts=starts, seed=9, job_id=app),
                              ex.walk(app, L, starts, seed=9, job_id=app))


def test_float_one_hop_distribution():
    n = 64
    w = np.array([0.001, 0.37, 1.0, 2.5, 3.25, 17.125, 999.9, 12345.678, 65535.5, 0.75], np.float32)
    src = np.zeros(len(w), np.uint32)
    dst = np.arange(1, len(w) + 1, dtype=np.uint32)
    g = Graph(float_weights=True)
    g.load_edges(src, dst, w, n)
    draws = 2_000_000
    out = g.walk(app=SAMPLING, starts=np.zeros(draws, np.uint32), seed=77)
    counts = np.bincount(out, minlength=n)[1:len(w) + 1].astype(np.float64)
    probs = w.astype(np.float64) / w.astype(np.float64).sum()
    assert _chisq(counts, probs) > ALPHA
    exact = fixed16(w).astype(np.float64)
    assert np.max(np.abs(exact / exact.sum() - probs) / probs) < 2.0 ** -16 / w.min() + 1e-12


@pytest.mark.parametrize("bad,status", [(0.0, "BINGO_ERR_ZERO_WEIGHT"), (-1.0, "BINGO_ERR_ZERO_WEIGHT"),
                                        (float("nan"), "BINGO_ERR_ZERO_WEIGHT"), (1e-6, "BINGO_ERR_ZERO_WEIGHT"),
                                        (65536.0, "BINGO_ERR_OUT_OF_RANGE"), (float("inf"), "BINGO_ERR_OUT_OF_RANGE")])
def test_float_weights_rejected_whole_batch(bad, status):
    n = 32
    src = np.array([0, 1, 2], np.uint32)
    dst = np.array([1, 2, 3], np.uint32)
    g = Graph(float_weights=True)
    g.load_edges(src, dst, np.array([1.5, 2.5, 3.5], np.float32), n)
    before = g.dump()
    with pytest.raises(BingoError) as e:
        g.insert_batch(np.array([4, 5], np.uint32), np.array([5, 6], np.uint32), np.array([2.0, bad], np.float32))
    assert e.value.name == status
    assert_exact_equal(g.dump(), before)


def test_integer_handle_refuses_float_weights():
    g = Graph()
    with pytest.raises(BingoError) as e:
        g.load_edges(np.array([0], np.uint32), np.array([1], np.uint32), np.array([1.5], np.float32), 4)
    assert e.value.name == "BINGO_ERR_INVALID_ARGUMENT"
