"""The CPU baseline's interleaved walk (several walks per thread in flight)
produces exactly the rows of the oracle's plain walk: DeepWalk and PPR, walk
lengths from 0 up, graphs with dead ends, tombstones and repeated starts."""
import numpy as np
import pytest

from bingo_b200 import gen
from oracle import pyoracle as po
from tests.helpers import workload

DEEPWALK, PPR = 0, 2


def _graph(scale, seed, dist, hi, rounds):
    n, src, dst, w, ops = workload(scale=scale, ef=8, seed=seed, dist=dist, lo=1, hi=hi, rounds=rounds,
                                   k_ins=300, k_del=900)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    for op in ops:
        if op[0] == "ins":
            ex.insert(*op[1:])
        else:
            ex.delete(*op[1:])
    return n, ex


@pytest.mark.parametrize("scale,seed,dist,hi,rounds", [(8, 3, gen.W_UNIFORM, 1024, 0),
                                                       (10, 4, gen.W_LOGUNIFORM, 2 ** 31, 3),
                                                       (12, 5, gen.W_ZIPF, 2 ** 24, 1)])
def test_interleaved_equals_plain(scale, seed, dist, hi, rounds):
    n, ex = _graph(scale, seed, dist, hi, rounds)
    rng = np.random.default_rng(seed)
    starts = np.concatenate([np.arange(n), rng.integers(0, n, 500)]).astype(np.uint32)
    for app, stop in ((DEEPWALK, 0.0125), (PPR, 0.0125), (PPR, 0.15), (PPR, 0.6)):
        for L in (0, 1, 2, 17, 80):
            a = ex.walk(app, L, starts, seed=77 + L, job_id=5, stop=stop)
            b = ex.walk_interleaved(app, L, starts, seed=77 + L, job_id=5, stop=stop)
            assert np.array_equal(a, b), (app, stop, L)


def test_interleaved_rejects_other_apps():
    ex = po.ExactGraph(4)
    with pytest.raises(ValueError):
        ex.walk_interleaved(1, 5, [0])
