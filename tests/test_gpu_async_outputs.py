"""Asynchronous handles copy host-bound walk rows out on a second stream
while later calls run; after bingo_sync every host buffer holds exactly the
rows a synchronous handle produces."""
import numpy as np
import pytest

from bingo_b200 import DEEPWALK, PPR, Graph
from tests.helpers import workload

pytestmark = pytest.mark.gpu


def test_overlapped_host_outputs_match_synchronous():
    n, src, dst, w, ops = workload(scale=12, ef=16, seed=91, rounds=3, k_ins=5000, k_del=4000)
    a, s = Graph(synchronous=False, node2vec=False), Graph(synchronous=True, node2vec=False)
    for g in (a, s):
        g.load_edges(src, dst, w, n)
    outs_a, outs_s, slots = [], [], []
    for r in range(6):
        app = DEEPWALK if r % 2 == 0 else PPR
        length = 40 + 8 * r  # growing outputs: the staging buffers are reallocated on the way
        if r < len(ops):
            op = ops[r]
            if op[0] == "ins":
                slot_a = a.insert_batch(*op[1:])  # host-bound slot ids, copied out beside the walk rows
                slot_s = s.insert_batch(*op[1:])
                slots.append((slot_a, slot_s))
            else:
                for g in (a, s):
                    g.delete_batch(*op[1:])
        for g, outs in ((a, outs_a), (s, outs_s)):
            out = np.full((n, length), -7, np.int32)
            g.walk(app=app, length=length, first=0, n_starts=n, seed=r, job_id=r, stop_prob=0.2, out=out)
            outs.append(out)
    a.sync()
    assert slots and all(np.array_equal(x, y) for x, y in slots)
    for x, y in zip(outs_a, outs_s):
        assert np.array_equal(x, y)
        assert (x != -7).all()
