"""Shared workload builders and state comparisons for the test suite."""
from __future__ import annotations

import numpy as np

from bingo_b200 import gen

MAXLOG = 16  # reference dense marker (include/api.h:11)


def workload(scale=10, ef=16, seed=11, dist=gen.W_UNIFORM, lo=1, hi=1024, s=1.2, rounds=2, k_ins=500, k_del=500):
    """An R-MAT graph plus `rounds` of (insert batch, delete batch)."""
    n = 1 << scale
    src, dst = gen.rmat(scale, ef, seed=seed)
    w = gen.weights(len(src), dist, lo, hi, s, seed=seed + 1)
    ug = gen.UpdateGen(n, src, dst, seed=seed + 2)
    ops = []
    for _ in range(rounds):
        ops.append(("ins",) + ug.inserts(k_ins, dist, lo, hi, s))
        ops.append(("del",) + ug.deletes(k_del))
    return n, src, dst, w, ops


def chisq_pvalue(counts, probs):
    """Pearson chi-square p-value of sampled counts against exact
    probabilities; bins whose expected count is below 5 are pooled into one
    (the chi-square approximation needs expected counts >= 5, and log-uniform
    weights give neighbours of probability ~1e-8). A draw of a
    zero-probability bin fails outright."""
    from scipy import stats
    counts = np.asarray(counts, np.float64)
    exp = np.asarray(probs, np.float64) * counts.sum()
    zero = exp == 0
    assert counts[zero].sum() == 0, "sampled a zero-probability neighbour"
    big = exp >= 5
    small = ~big & ~zero
    obs_b, exp_b = list(counts[big]), list(exp[big])
    if small.any():
        obs_b.append(counts[small].sum())
        exp_b.append(exp[small].sum())
        if exp_b[-1] < 5 and len(exp_b) > 1:  # fold a still-small pool into the smallest bin
            j = int(np.argmin(exp_b[:-1]))
            obs_b[j] += obs_b.pop()
            exp_b[j] += exp_b.pop()
    return stats.chisquare(np.array(obs_b), np.array(exp_b)).pvalue


def csr_offsets(counts):
    off = np.zeros(len(counts) + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return off


def assert_exact_equal(a: dict, b: dict, what=""):
    for k in ["ecnt", "live", "ev", "ew", "gcnt", "mslot", "mv", "mbp", "am", "athr", "aT", "aown", "aalias"]:
        x, y = a[k], b[k]
        assert x.shape == y.shape, f"{what}{k}: shape {x.shape} != {y.shape}"
        if not np.array_equal(x, y):
            bad = np.nonzero(x != y)[0]
            raise AssertionError(f"{what}{k}: {len(bad)} mismatches, first at {bad[:5]}: {x[bad[:5]]} vs {y[bad[:5]]}")


def check_exact_invariants(d: dict, n: int):
    """Internal consistency of an exact-semantics dump."""
    eoff = csr_offsets(d["ecnt"].astype(np.int64))
    gcnt = d["gcnt"].astype(np.int64)
    moff = csr_offsets(gcnt)
    ew = d["ew"]
    # member neighbour equals its slot's neighbour; back-pointer equals position
    vert_of_member = np.repeat(np.repeat(np.arange(n), 32), gcnt)
    bit_of_member = np.repeat(np.tile(np.arange(32), n), gcnt)
    pos = np.arange(len(d["mslot"])) - np.repeat(moff[:-1], gcnt)
    gslot = eoff[vert_of_member] + d["mslot"].astype(np.int64)
    assert np.all(d["mslot"] < d["ecnt"][vert_of_member])
    assert np.array_equal(d["mv"], d["ev"][gslot])
    assert np.array_equal(d["mbp"].astype(np.int64), pos)
    assert np.all((ew[gslot] >> bit_of_member.astype(np.uint32)) & 1)
    # group counts equal the live popcount per bit
    vert_of_slot = np.repeat(np.arange(n), d["ecnt"].astype(np.int64))
    for k in range(32):
        has = ((ew >> np.uint32(k)) & 1).astype(np.int64)
        cnt = np.bincount(vert_of_slot, weights=has, minlength=n).astype(np.int64)
        assert np.array_equal(cnt, gcnt.reshape(n, 32)[:, k]), f"bit {k} count"
    live = np.bincount(vert_of_slot, weights=(ew != 0), minlength=n).astype(np.int64)
    assert np.array_equal(live, d["live"].astype(np.int64))
    # alias: one slot per nonzero group, exact mass invariant
    nz = (gcnt.reshape(n, 32) > 0).sum(1)
    assert np.array_equal(nz, d["am"].astype(np.int64))
    aoff = csr_offsets(d["am"].astype(np.int64))
    mass = gcnt.reshape(n, 32).astype(object) * (1 << np.arange(32)).astype(object)
    for u in np.nonzero(nz)[0][:2000]:
        m = int(nz[u])
        a0 = aoff[u]
        T = int(sum(mass[u]))
        contrib = [0] * 32
        for j in range(m):
            thr = int(d["athr"][a0 + j])
            assert int(d["aT"][a0 + j]) == T
            contrib[d["aown"][a0 + j]] += thr
            contrib[d["aalias"][a0 + j]] += T - thr
        for k in range(32):
            assert contrib[k] == int(mass[u][k]) * m


def compare_exact_vs_ref(ex: dict, rf: dict, n: int, check_alias_tol=None):
    """The reference's structures (sparse-group member sequences, back-pointers,
    float masses below LOGT, slots, weights, capacities) against the exact
    dump of the same inputs. Returns the max |p_ref - p_exact| over groups."""
    assert np.array_equal(ex["ecnt"], rf["ecnt"]), "slot counts"
    assert np.array_equal(ex["ev"], rf["ev"]), "slot neighbours"
    assert np.array_equal(ex["ew"].astype(np.float32), rf["ew"]), "slot weights / tombstones"
    logt = rf["logt"].astype(np.int64)
    bits = rf["bits"].astype(np.int64)
    toff = csr_offsets(logt)
    boff = csr_offsets(bits)
    goff = csr_offsets(rf["gsz"].astype(np.int64))
    gcnt = ex["gcnt"].astype(np.int64)
    moff = csr_offsets(gcnt)
    aoff_r = csr_offsets(rf["asz"].astype(np.int64))
    worst = 0.0
    for u in range(n):
        L = int(logt[u])
        for j in range(L):
            tp = int(rf["grouptp"][toff[u] + j])
            c = int(gcnt[u * 32 + j])
            assert rf["num"][toff[u] + j] == np.float32(c * (1 << j)), f"num[{u}][{j}]"
            if tp != MAXLOG:
                gi = boff[u] + tp
                ref_list = rf["members"][goff[gi]:goff[gi + 1]]
                ex_list = ex["mslot"][moff[u * 32 + j]:moff[u * 32 + j] + c]
                assert np.array_equal(ref_list, ex_list), f"group list u={u} bit={j}"
                assert np.array_equal(rf["midx"][goff[gi]:goff[gi + 1]], np.arange(len(ref_list))), f"idx u={u}"
        if check_alias_tol is not None and rf["asz"][u]:
            a0, a1 = aoff_r[u], aoff_r[u + 1]
            sz = a1 - a0
            pr = np.zeros(32)
            for e in range(a0, a1):
                p = min(1.0, max(0.0, float(rf["ap"][e])))
                if rf["aa"][e] >= 0:
                    pr[rf["aa"][e]] += p / sz
                if rf["ab"][e] >= 0:
                    pr[rf["ab"][e]] += (1 - p) / sz
            mass = np.array([gcnt[u * 32 + k] * float(1 << k) if k < L else 0.0 for k in range(32)])
            if mass.sum() > 0:
                worst = max(worst, float(np.abs(pr - mass / mass.sum()).max()))
    if check_alias_tol is not None:
        assert worst <= check_alias_tol, f"reference alias deviates by {worst}"
    return worst
