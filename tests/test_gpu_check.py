"""Store check (bingo_check): clean on every store the update kernels
produce, with totals equal to the oracle's; and a snapshot whose content
breaks an invariant (edited here on the CPU, checksum recomputed) is refused
with BINGO_ERR_CORRUPT naming the damaged vertex and the kind of damage,
before any kernel but the check reads it."""
import struct

import numpy as np
import pytest

from bingo_b200 import DEEPWALK, BingoError, Graph, gen
from oracle import pyoracle as po
from tests.helpers import assert_exact_equal, workload

pytestmark = pytest.mark.gpu

EXTENT, COUNT, MEMBER, ALIAS, HASH, RANGE = 1, 2, 4, 8, 16, 32


def _expected(d):
    live_w = d["ew"][d["ew"] != 0].astype(np.uint64)
    return dict(live_edges=int(d["live"].sum()), weight_sum=int(live_w.sum()), members=int(d["gcnt"].sum()),
                alias_slots=int(d["am"].sum()))


def _assert_clean(g, ex):
    rep = g.check()
    assert rep["bad_vertices"] == 0 and rep["kinds"] == 0 and rep["first_bad"] == 0xFFFFFFFF
    assert rep["vertices"] == g.n
    want = _expected(ex.dump())
    assert {k: rep[k] for k in want} == want


@pytest.mark.parametrize("node2vec", [False, True])
def test_clean_after_every_batch(node2vec):
    n, src, dst, w, ops = workload(scale=12, ef=10, seed=5, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 31, rounds=3,
                                   k_ins=5000, k_del=4000)
    g, ex = Graph(node2vec=node2vec), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    _assert_clean(g, ex)
    for op in ops:
        if op[0] == "ins":
            g.insert_batch(*op[1:])
            ex.insert(*op[1:])
        else:
            g.delete_batch(*op[1:])
            ex.delete(*op[1:])
        _assert_clean(g, ex)
    # delete by pair, then the same pairs again (all absent: skipped)
    live = ex.dump()
    us = np.repeat(np.arange(n, dtype=np.uint32), live["ecnt"])
    keep = live["ew"] != 0
    pick = np.flatnonzero(keep)[::7][:3000]
    u, v = us[pick], live["ev"][pick]
    g.delete_pairs(u, v)
    ex.delete_pairs(u, v)
    _assert_clean(g, ex)
    assert_exact_equal(g.dump(), ex.dump())


def test_check_of_empty_and_edgeless_graphs():
    g = Graph(node2vec=True)
    g.load_edges(np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32), 100)
    rep = g.check()
    assert rep["bad_vertices"] == 0 and rep["live_edges"] == 0 and rep["alias_slots"] == 0
    with pytest.raises(BingoError) as e:
        Graph().check()
    assert e.value.name == "BINGO_ERR_NOT_LOADED"


# ---------------------------------------------------------------- snapshots
# File layout: 96-byte header (magic, version, node2vec, n, bits,
# rec_bytes[4], top[5], payload_bytes, checksum), then VertexRec[n],
# VertexMeta[n], GroupDesc[n][32], the used part of the member, edge,
# back-pointer, alias and adjacency arenas, and the members' back-pointer indices.
HDR = struct.Struct("<8s4I4I5QQQ")
MASK = (1 << 64) - 1
CHUNK = 64 << 20


def _snapsum(parts):
    """The file's checksum: word-wise multiply-xor over each part, in
    64 MiB pieces, tail bytes folded one by one."""
    h = 0x9E3779B97F4A7C15
    prime = 0x100000001B3
    for p in parts:
        for o in range(0, len(p), CHUNK):
            b = p[o:o + CHUNK]
            nw = len(b) // 8
            for x in np.frombuffer(b[:nw * 8], dtype="<u8").tolist():
                h = ((h ^ x) * prime) & MASK
                h ^= h >> 29
            for c in b[nw * 8:]:
                h = ((h ^ c) * prime) & MASK
    return h


class Snap:
    def __init__(self, raw: bytes):
        f = HDR.unpack_from(raw, 0)
        self.magic, self.version, self.node2vec, self.n, self.bits = f[:5]
        self.rec = f[5:9]
        self.top = list(f[9:14])
        self.payload, self.checksum = f[14], f[15]
        n = self.n
        sizes = [n * self.rec[0], n * self.rec[1], n * 32 * self.rec[2], self.top[0] * 4, self.top[1] * 16,
                 self.top[2] * 4, self.top[3] * self.rec[3], self.top[4] * 16, self.top[0] * 4]
        assert sum(sizes) == self.payload and len(raw) == HDR.size + self.payload
        self.parts, o = [], HDR.size
        for s in sizes:
            self.parts.append(bytearray(raw[o:o + s]))
            o += s
        assert _snapsum(self.parts) == self.checksum

    def names(self):
        return dict(vrec=0, meta=1, gdesc=2, member=3, edge=4, bp=5, alias=6, hash=7, gs=8)

    def u32(self, part, idx, field=0, stride=None):
        p = self.parts[self.names()[part]]
        return struct.unpack_from("<I", p, idx * (stride or 4) + field * 4)[0]

    def set_u32(self, part, byte_off, value):
        struct.pack_into("<I", self.parts[self.names()[part]], byte_off, value)

    def u64(self, part, byte_off):
        return struct.unpack_from("<Q", self.parts[self.names()[part]], byte_off)[0]

    def set_u64(self, part, byte_off, value):
        struct.pack_into("<Q", self.parts[self.names()[part]], byte_off, value & MASK)

    # records
    def vrec(self, u):  # aoff, m, hoff, hmask
        return struct.unpack_from("<4I", self.parts[0], u * self.rec[0])

    def meta(self, u):  # eoff, bpoff, ecnt, ecap, bpcnt, bpcap, live, acap, hkeys, hcap
        return struct.unpack_from("<QQ8I", self.parts[1], u * self.rec[1])

    def group(self, u, k):  # base (4-entry units), cnt, capacity (derived, as the engine derives it)
        base1, word = struct.unpack_from("<2I", self.parts[2], (u * 32 + k) * self.rec[2])
        cnt, roomy = word & 0x7FFFFFFF, word >> 31
        cap = 0
        if base1:
            cap = 4
            while cap < cnt:
                cap <<= 1
            cap <<= roomy
        return (base1 - 1 if base1 else 0), cnt, cap

    def edge(self, i):  # v, w, ebp
        return struct.unpack_from("<3I", self.parts[4], i * 16)

    def write(self, path):
        head = HDR.pack(self.magic, self.version, self.node2vec, self.n, self.bits, *self.rec, *self.top,
                        self.payload, _snapsum(self.parts))
        path.write_bytes(head + b"".join(bytes(p) for p in self.parts))


@pytest.fixture(scope="module", params=[False, True], ids=["plain", "node2vec"])
def saved(request, tmp_path_factory):
    node2vec = request.param
    n, src, dst, w, ops = workload(scale=10, ef=8, seed=21, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 20, rounds=1,
                                   k_ins=800, k_del=600)
    g, ex = Graph(node2vec=node2vec), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    for op in ops:
        if op[0] == "ins":
            g.insert_batch(*op[1:])
            ex.insert(*op[1:])
        else:
            g.delete_batch(*op[1:])
            ex.delete(*op[1:])
    path = tmp_path_factory.mktemp("snap") / f"g{int(node2vec)}.snap"
    g.save(path)
    return node2vec, path, ex


def _vertex(s, pred):
    for u in range(s.n):
        if pred(u):
            return u
    raise AssertionError("no vertex fits")


def _refused(node2vec, path, bad, ex, u, kinds):
    h = Graph(node2vec=node2vec)
    with pytest.raises(BingoError) as e:
        h.restore(bad)
    assert e.value.name == "BINGO_ERR_CORRUPT"
    assert f"first {u}, kinds {kinds}" in str(e.value), str(e.value)
    with pytest.raises(BingoError) as e2:  # no graph after a refused restore
        h.walk(app=DEEPWALK, length=4, starts=np.zeros(2, np.uint32))
    assert e2.value.name == "BINGO_ERR_NOT_LOADED"
    h.restore(path)  # the undamaged file restores into the same handle
    assert_exact_equal(h.dump(), ex.dump())
    assert h.check()["bad_vertices"] == 0


def test_snapshot_round_trip_is_clean(saved):
    node2vec, path, ex = saved
    s = Snap(path.read_bytes())
    assert s.node2vec == int(node2vec)
    h = Graph(node2vec=node2vec)
    h.restore(path)
    rep = h.check()
    assert rep["bad_vertices"] == 0
    assert {k: rep[k] for k in ("live_edges", "weight_sum", "members", "alias_slots")} == _expected(ex.dump())


def test_alias_threshold_damage(saved, tmp_path):
    node2vec, path, ex = saved
    s = Snap(path.read_bytes())
    # a slot that splits its mass between two groups
    def split_slot(u):
        aoff, m = s.vrec(u)[:2]
        return any(s.u64("alias", (aoff + j) * s.rec[3]) < s.u64("alias", (aoff + j) * s.rec[3] + 8)
                   for j in range(m))
    u = _vertex(s, lambda x: s.vrec(x)[1] >= 2 and split_slot(x))
    aoff, m = s.vrec(u)[:2]
    j = next(j for j in range(m) if s.u64("alias", (aoff + j) * s.rec[3]) < s.u64("alias", (aoff + j) * s.rec[3] + 8))
    off = (aoff + j) * s.rec[3]
    s.set_u64("alias", off, s.u64("alias", off) + 1)
    bad = tmp_path / "alias.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, ALIAS)


def test_member_neighbour_damage(saved, tmp_path):
    node2vec, path, ex = saved
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.group(x, 0)[1] > 0 or any(s.group(x, k)[1] for k in range(32)))
    k = next(k for k in range(32) if s.group(u, k)[1])
    base = s.group(u, k)[0]
    v = s.u32("member", base * 4)
    s.set_u32("member", base * 16, (v + 1) % s.n)
    bad = tmp_path / "member.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, MEMBER)


def test_neighbour_out_of_range(saved, tmp_path):
    node2vec, path, ex = saved
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.meta(x)[6] > 0)
    eoff, ecnt = s.meta(u)[0], s.meta(u)[2]
    slot = next(i for i in range(ecnt) if s.edge(eoff + i)[1])
    s.set_u32("edge", (eoff + slot) * 16, s.n)  # its members still hold the old id
    bad = tmp_path / "range.snap"
    s.write(bad)
    # the members disagree with the slot; with the adjacency index the new id is also missing from it
    _refused(node2vec, path, bad, ex, u, RANGE | MEMBER | (HASH if node2vec else 0))


def test_count_damage(saved, tmp_path):
    node2vec, path, ex = saved
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.meta(x)[6] > 0)
    s.set_u32("meta", u * s.rec[1] + 32, s.meta(u)[6] - 1)  # live
    bad = tmp_path / "count.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, COUNT)


def test_extent_damage(saved, tmp_path):
    node2vec, path, ex = saved
    # a slot count above the vertex's capacity
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.meta(x)[3] > 0)
    s.set_u32("meta", u * s.rec[1] + 16, s.meta(u)[3] + 1)  # ecnt = ecap + 1
    bad = tmp_path / "extent1.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, EXTENT)
    # an alias table that starts past the used part of the alias arena
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.meta(x)[7] > 0)
    s.set_u32("vrec", u * s.rec[0], s.top[3])
    bad = tmp_path / "extent2.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, EXTENT)
    # a group list that reaches past the used part of the member arena
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.group(x, 0)[2] > 0)
    s.set_u32("gdesc", u * 32 * s.rec[2], s.top[0] // 4 + 1)  # list base = the end of the used part
    bad = tmp_path / "extent3.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, EXTENT)


def test_adjacency_damage(saved, tmp_path):
    node2vec, path, ex = saved
    if not node2vec:
        pytest.skip("adjacency index only on node2vec handles")
    s = Snap(path.read_bytes())
    u = _vertex(s, lambda x: s.vrec(x)[3] > 0 and s.meta(x)[6] > 0)
    hoff, hmask = s.vrec(u)[2:]
    h = next(i for i in range(hmask + 1) if struct.unpack_from("<i", s.parts[7], (hoff + i) * 16)[0] != -1)
    off = (hoff + h) * 16 + 8
    s.set_u64("hash", off, s.u64("hash", off) + 3)
    bad = tmp_path / "hash.snap"
    s.write(bad)
    _refused(node2vec, path, bad, ex, u, HASH)


def test_large_vertex_damage(tmp_path):
    """A vertex with more than 4096 group members is checked by a whole CTA;
    damage there is reported once, merged with the vertex's other results."""
    n, src, dst, w, _ = workload(scale=13, ef=16, seed=8, dist=gen.W_LOGUNIFORM, lo=1, hi=2 ** 31, rounds=0)
    g, ex = Graph(node2vec=False), po.ExactGraph(n)
    g.load_edges(src, dst, w, n)
    ex.load(src, dst, w)
    path = tmp_path / "big.snap"
    g.save(path)
    s = Snap(path.read_bytes())
    members = lambda x: sum(s.group(x, k)[1] for k in range(32))  # noqa: E731
    u = _vertex(s, lambda x: members(x) > 4096)
    # the last member of the vertex's highest group: far from the start of its range
    k = max(k for k in range(32) if s.group(u, k)[1])
    base, cnt = s.group(u, k)[:2]
    v = s.u32("member", base * 4 + cnt - 1)
    s.set_u32("member", (base * 4 + cnt - 1) * 4, (v + 1) % s.n)
    bad = tmp_path / "big_member.snap"
    s.write(bad)
    _refused(False, path, bad, ex, u, MEMBER)
    # the same member damage plus a live-count error on the same vertex: one
    # bad vertex carrying both kinds
    s.set_u32("meta", u * s.rec[1] + 32, s.meta(u)[6] - 1)
    s.write(bad)
    h = Graph(node2vec=False)
    with pytest.raises(BingoError) as e:
        h.restore(bad)
    assert e.value.name == "BINGO_ERR_CORRUPT"
    assert f"1 vertices, first {u}, kinds {MEMBER | COUNT}" in str(e.value), str(e.value)
