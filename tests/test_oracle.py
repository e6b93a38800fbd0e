"""CPU oracle checks (no GPU): Philox known answers, the integer alias
invariant, the exact semantics against the reference-literal state machine,
and the golden dumps produced by the reference's own CUDA build."""
import glob
import json
import os

import numpy as np
import pytest

from bingo_b200 import gen
from oracle import pyoracle as po
from tests.helpers import check_exact_invariants, compare_exact_vs_ref, workload

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors (Salmon et al., SC'11).
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kat:
        assert list(po.philox(ctr, key)) == want


def _alias_check(cnt):
    mass = [(c << k) if c else 0 for k, c in enumerate(cnt)]
    m, thr, T, own, al = po.alias_build(mass)
    nz = [k for k in range(32) if mass[k]]
    assert m == len(nz)
    if not m:
        return
    tot = sum(mass)
    contrib = [0] * 32
    for j in range(m):
        assert int(T[j]) == tot and int(thr[j]) <= tot
        assert own[j] == nz[j]
        contrib[own[j]] += int(thr[j])
        contrib[al[j]] += tot - int(thr[j])
    assert contrib == [x * m for x in mass]


def test_alias_invariant_exhaustive_small():
    import itertools
    for cnt3 in itertools.product(range(4), repeat=3):
        for bits in [(0, 1, 2), (0, 5, 31), (3, 4, 30)]:
            cnt = [0] * 32
            for b, c in zip(bits, cnt3):
                cnt[b] = c
            _alias_check(cnt)


def test_alias_invariant_random():
    rng = np.random.default_rng(5)
    for _ in range(3000):
        cnt = [int(x) for x in rng.choice([0, 0, 0, 1, 2, 3, 17, 1000, 2 ** 20], size=32)]
        if sum(c << k for k, c in enumerate(cnt)) >= 2 ** 64:
            continue
        _alias_check(cnt)


def test_alias_extremes():
    _alias_check([0] * 31 + [2 ** 32 - 1])          # one group at bit 31
    _alias_check([2 ** 31] + [0] * 30 + [2 ** 31 - 1])  # 2^31 units vs ~2^62
    _alias_check([1] * 32)


@pytest.mark.parametrize("seed,dist,lo,hi", [(11, gen.W_UNIFORM, 1, 1024), (21, gen.W_UNIFORM, 1, 65535),
                                             (31, gen.W_LOGUNIFORM, 1, 2 ** 16), (41, gen.W_UNIFORM, 1, 3)])
def test_exact_matches_reference_literal(seed, dist, lo, hi):
    """Sparse-group member sequences, back-pointers, masses, slots and
    tombstones of the exact semantics equal the reference state machine."""
    n, src, dst, w, ops = workload(scale=9, ef=12, seed=seed, dist=dist, lo=lo, hi=hi, rounds=3, k_ins=400,
                                   k_del=400)
    ex, rf = po.ExactGraph(n), po.RefGraph(n)
    ex.load(src, dst, w)
    rf.load(src, dst, w)
    worst = compare_exact_vs_ref(ex.dump(), rf.dump(), n, check_alias_tol=5e-3)
    for op in ops:
        if op[0] == "ins":
            ex.insert(*op[1:])
            rf.insert(*op[1:])
        else:
            assert ex.delete(*op[1:]) == 0
            rf.delete(*op[1:])
        d = ex.dump()
        check_exact_invariants(d, n)
        worst = max(worst, compare_exact_vs_ref(d, rf.dump(), n, check_alias_tol=5e-3))


def test_exact_delete_rejects_bad_slots():
    n, src, dst, w, _ = workload(scale=6, ef=4, seed=3, rounds=0)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    u0 = int(src[0])
    # out of range slot, then double delete of slot 0 within one batch
    assert ex.delete([u0], [10 ** 6]) == 1
    assert ex.delete([u0, u0], [0, 0]) == 1
    check_exact_invariants(ex.dump(), n)


def test_walk_rows_follow_edges():
    n, src, dst, w, _ = workload(scale=8, ef=8, seed=5, rounds=0)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    adj = set(zip(src.tolist(), dst.tolist()))
    starts = np.arange(n, dtype=np.uint32)
    for app in (0, 1, 2):
        rows = ex.walk(app, 20, starts, seed=9, job_id=app, stop=0.2)
        assert np.array_equal(rows[:, 0], starts)
        for r in rows[:50]:
            for a, b in zip(r[:-1], r[1:]):
                if b < 0:
                    break
                assert (int(a), int(b)) in adj
            k = np.argmax(r < 0) if (r < 0).any() else len(r)
            assert (r[k:] == -1).all()


def test_walk_determinism_and_counter_independence():
    n, src, dst, w, _ = workload(scale=8, ef=8, seed=6, rounds=0)
    ex = po.ExactGraph(n)
    ex.load(src, dst, w)
    starts = np.arange(n, dtype=np.uint32)
    a = ex.walk(0, 30, starts, seed=1)
    b = ex.walk(0, 30, starts, seed=1)
    c = ex.walk(0, 30, starts, seed=2)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    # walk i depends only on (seed, job, i): a subset of starts reproduces rows
    sub = ex.walk(0, 30, starts[:10], seed=1)
    assert np.array_equal(sub, a[:10])


def _golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def test_golden_fixtures_present():
    assert _golden_cases(), "reference golden fixtures missing (tests/golden/make_golden.py)"


@pytest.mark.parametrize("path", _golden_cases(), ids=os.path.basename)
def test_reference_literal_matches_reference_dumps(path):
    """Pins the CPU restatement to the reference's own CUDA build: the state
    the reference binary dumped after load and after every batch equals the
    reference-literal oracle's, bit for bit (float masses and alias included)."""
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    n = meta["n"]
    rf = po.RefGraph(n, meta["rate"])
    ex = po.ExactGraph(n)
    rf.load(z["src"], z["dst"], z["w"])
    ex.load(z["src"], z["dst"], z["w"])
    steps = meta["ops"]
    for i, op in enumerate(["load"] + steps):
        if op == "ins":
            args = (z[f"op{i}_a"], z[f"op{i}_b"], z[f"op{i}_c"])
            rf.insert(*args)
            ex.insert(*args)
        elif op == "del":
            args = (z[f"op{i}_a"], z[f"op{i}_b"])
            rf.delete(*args)
            ex.delete(*args)
        mine = rf.dump()
        for k in po.REF_DUMP_FIELDS:
            want = z[f"dump{i}_{k}"]
            assert np.array_equal(mine[k], want), f"{os.path.basename(path)} step {i} ({op}) field {k}"
        compare_exact_vs_ref(ex.dump(), mine, n)


def test_reference_rmat14_digests():
    """The small DeepWalk workload (R-MAT 14, uniform [1,1024], 10K + 10K): the
    reference binary's dumps after load, insert and delete, stored as SHA-256
    digests, equal the reference-literal oracle replaying the same inputs."""
    import hashlib
    import importlib.util
    rec = json.load(open(os.path.join(GOLDEN, "ref_rmat14_digest.json")))
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    case = mg.rmat14_case()
    dig = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    for k in ("src", "dst", "w"):
        assert dig(case[k]) == rec["inputs"][k], f"input {k} drifted from the fixture"
    rf = po.RefGraph(case["n"], case["rate"])
    rf.load(case["src"], case["dst"], case["w"])
    dumps = [rf.dump()]
    for op in case["ops"]:
        (rf.insert if op[0] == "ins" else rf.delete)(*op[1:])
        dumps.append(rf.dump())
    assert len(dumps) == len(rec["dumps"])
    for i, (mine, want) in enumerate(zip(dumps, rec["dumps"])):
        for k in po.REF_DUMP_FIELDS:
            assert dig(mine[k]) == want[k], f"rmat14 dump {i} field {k}"


def test_oracle_delete_pairs_rank_semantics():
    """r-th repeat of (u, v) takes the r-th lowest live slot; extra repeats and
    absent pairs are rejected without touching the graph."""
    ex = po.ExactGraph(4)
    src = np.array([0, 0, 0, 0, 1], np.uint32)
    dst = np.array([1, 2, 1, 1, 2], np.uint32)
    w = np.array([3, 5, 7, 9, 1], np.uint32)
    ex.load(src, dst, w)
    ex.delete(np.array([0], np.uint32), np.array([2], np.uint32))  # slot 2 (0->1) is now a tombstone
    bad, slots = ex.delete_pairs(np.array([0, 1, 0, 0, 2], np.uint32), np.array([1, 2, 1, 1, 3], np.uint32))
    assert list(slots) == [0, 0, 3, 0xFFFFFFFF, 0xFFFFFFFF]
    assert bad == 2
    d = ex.dump()
    assert d["live"][0] == 1 and d["live"][1] == 0
