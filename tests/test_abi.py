"""The C ABI library loads and exports every symbol include/*.h declares;
host-only pieces (generators) behave; no GPU compute is called here."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import bingo_b200
from bingo_b200 import gen
from bingo_b200._lib import SIGNATURES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(bingo_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = bingo_b200.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for name in sorted(names):
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
        assert name in SIGNATURES, f"{name} has no ctypes signature"


def test_no_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from bingo_b200 import BingoError, Graph
    with pytest.raises(BingoError) as e:
        Graph()
    assert e.value.name == "BINGO_ERR_NO_DEVICE"


def test_rmat_deterministic_and_clean():
    a = gen.rmat(12, 8, seed=3)
    b = gen.rmat(12, 8, seed=3)
    c = gen.rmat(12, 8, seed=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[1], c[1])
    s, d = a
    assert (s != d).all()
    key = s.astype(np.int64) << 32 | d
    assert (np.diff(key) > 0).all()  # sorted, no duplicates
    deg = np.bincount(s, minlength=1 << 12)
    assert deg.max() > 20 * deg.mean()  # skewed


def test_weight_distributions():
    u = gen.weights(200000, gen.W_UNIFORM, 1, 1024, seed=1)
    assert u.min() == 1 and u.max() == 1024 and abs(u.mean() - 512.5) < 5
    lg = gen.weights(200000, gen.W_LOGUNIFORM, 1, 2 ** 20, seed=1)
    assert lg.min() >= 1 and lg.max() < 2 ** 20
    frac = np.histogram(np.log2(lg.astype(np.float64) + 0.5), bins=20, range=(0, 20))[0] / len(lg)
    assert frac[5:].std() < 0.01  # flat in log scale
    z = gen.weights(200000, gen.W_ZIPF, 1, 2 ** 24 - 1, 1.2, seed=1)
    hn = sum(k ** -1.2 for k in range(1, 100000)) + (100000 ** -0.2 - (2 ** 24) ** -0.2) / 0.2
    assert abs((z == 1).mean() - 1 / hn) < 0.005
    assert abs((z == 2).mean() - 2 ** -1.2 / hn) < 0.005


def test_update_generator_tracks_slots():
    n = 1 << 10
    s, d = gen.rmat(10, 8, seed=5)
    ug = gen.UpdateGen(n, s, d, seed=6)
    live0 = ug.live
    i_s, i_d, i_w = ug.inserts(3000)
    pairs = set(zip(s.tolist(), d.tolist()))
    assert not any((a, b) in pairs for a, b in zip(i_s.tolist(), i_d.tolist()))
    assert len(set(zip(i_s.tolist(), i_d.tolist()))) == 3000
    assert (i_s != i_d).all() and (i_w >= 1).all()
    u, slot = ug.deletes(2000)
    assert len(set(zip(u.tolist(), slot.tolist()))) == 2000
    deg = np.bincount(np.concatenate([s, i_s]), minlength=n)
    assert (slot < deg[u]).all()
    assert ug.live == live0 + 3000 - 2000
