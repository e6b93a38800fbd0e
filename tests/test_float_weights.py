"""Float-weight mode on the host: the 16.16 fixed-point conversion
(bingo_weights_to_fixed16) rounds half to even and rejects what the device
rejects."""
import numpy as np

from bingo_b200 import fixed16


def test_fixed16_rounding_and_limits():
    q = 2.0 ** -16
    w = np.array([1.0, 0.5, 1.5 * q, 2.5 * q, 0.5 * q, 0.49 * q, 65535.99609375, 65536.0, 0.0, -3.0,
                  np.nan, np.inf, 1234.5678], np.float32)
    out = fixed16(w)
    assert out.tolist()[:6] == [65536, 32768, 2, 2, 0, 0]  # 1.5 -> 2 and 2.5 -> 2: half to even
    assert out[6] == 4294967040
    assert (out[7:12] == 0).all()
    assert out[12] == int(np.rint(np.float32(1234.5678) * np.float32(65536)))


def test_fixed16_matches_numpy_restatement():
    rng = np.random.default_rng(4)
    w = np.exp(rng.uniform(np.log(1e-5), np.log(65535.9), size=200_000)).astype(np.float32)
    ref = np.rint(w * np.float32(65536)).astype(np.uint64)
    ref[(ref == 0) | (w >= 65536)] = 0
    assert np.array_equal(fixed16(w), ref.astype(np.uint32))
