"""The reference's own inputs on the host: the edge-list reader and the
driver's load weights (include/graph.cuh:22-51, include/api.h:29-30)."""
import numpy as np
import pytest

from bingo_b200 import gen


def _write(tmp_path, text, name="g.txt"):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return str(p)


def test_reader_keeps_file_order_and_skips_comments(tmp_path):
    p = _write(tmp_path, "# SNAP header\n% another\n0 1\n2\t0\r\n\n  5 5\n1 2 3 4\n0 1")
    src, dst, n = gen.read_edge_list(p)
    assert src.tolist() == [0, 2, 5, 1, 3, 0]
    assert dst.tolist() == [1, 0, 5, 2, 4, 1]
    assert n == 6


@pytest.mark.parametrize("text,what", [("0 1\n2 x\n", "malformed"), ("0 1\n2\n", "malformed"),
                                       ("0 4294967295\n", "above"), ("1 -2\n", "malformed")])
def test_reader_rejects_bad_input(tmp_path, text, what):
    with pytest.raises(ValueError, match=what):
        gen.read_edge_list(_write(tmp_path, text))


def test_reader_missing_file(tmp_path):
    with pytest.raises(ValueError, match="cannot open"):
        gen.read_edge_list(str(tmp_path / "absent.txt"))


def test_reader_large_round_trip(tmp_path):
    src, dst = gen.rmat(14, 8, seed=4)
    p = tmp_path / "big.txt"
    np.savetxt(p, np.stack([src, dst], 1), fmt="%d")
    s2, d2, n = gen.read_edge_list(str(p))
    assert np.array_equal(s2, src) and np.array_equal(d2, dst)
    assert n == int(max(src.max(), dst.max())) + 1


def _ref_weights(src, dst, n, pow03):
    d = np.bincount(src, minlength=n).astype(np.int64)[dst]
    if pow03:
        b = np.power(d.astype(np.float64), 0.3).astype(np.float32)
    else:
        b = d.astype(np.float32)
    return (b + np.float32(1)).astype(np.uint32)


def test_driver_weights_match_the_reference_formula():
    src, dst = gen.rmat(13, 16, seed=9)
    n = 1 << 13
    for kind, pow03 in ((gen.DRIVER_DEGREE, False), (gen.DRIVER_DEGREE_POW03, True), (gen.DRIVER_AUTO, False)):
        assert np.array_equal(gen.driver_weights(src, dst, n, kind), _ref_weights(src, dst, n, pow03))
    assert (gen.driver_weights(src, dst, n) >= 1).all()
    with pytest.raises(ValueError):
        gen.driver_weights(src, dst, 10)
