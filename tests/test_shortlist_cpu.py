"""The shortlist network's CPU restatement (the checker of its GPU training kernels): bf16 rounding and analytic
gradients against finite differences; the initial weights are seeded."""
import numpy as np

import shortlist_ref as R
from av1gpu_b200 import shortlist as SL


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, -3.14159, 65504.0, 1e-30], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0078125 or r[1] == 1.0   # halfway cases go to even
    assert abs(r[3] - (-3.140625)) < 1e-9
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8 + 1e-38)


def test_restated_gradients_by_finite_differences():
    rng = np.random.default_rng(0)
    n = 16
    X = rng.standard_normal((n, SL.N_IN))
    y = rng.integers(0, SL.N_MODES, n)
    w1, b1, w2, b2 = [a.astype(np.float64) for a in SL.init_weights(2)]
    b1 = b1 + 0.05
    # without the bf16 rounding of the hidden layer the restatement's gradients are exact: compare in float64
    def loss(w1_, b1_, w2_, b2_):
        h = np.maximum(X @ w1_.T + b1_, 0)
        s = h @ w2_.T + b2_
        z = s[:, :13] - s[:, :13].max(1, keepdims=True)
        return float(-(z[np.arange(n), y] - np.log(np.exp(z).sum(1))).mean())
    h = np.maximum(X @ w1.T + b1, 0)
    R_bf16 = R.bf16
    try:
        R.bf16 = lambda a: np.asarray(a, np.float64)
        (gw1, gb1, gw2, gb2), l, _ = R.grads(X, y, w1, b1, w2, b2)
    finally:
        R.bf16 = R_bf16
    assert abs(l - loss(w1, b1, w2, b2)) < 1e-12
    eps = 1e-6
    for (arr, g, idx) in ((w1, gw1, (5, 17)), (b1, gb1, (9,)), (w2, gw2, (3, 40)), (b2, gb2, (2,))):
        a0 = arr[idx]
        arr[idx] = a0 + eps
        lp = loss(w1, b1, w2, b2)
        arr[idx] = a0 - eps
        lm = loss(w1, b1, w2, b2)
        arr[idx] = a0
        assert abs((lp - lm) / (2 * eps) - g[idx]) < 1e-6


def test_init_weights_seeded():
    a, b = SL.init_weights(7), SL.init_weights(7)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert a[0].shape == (SL.N_HID, SL.N_IN) and a[2].shape == (SL.N_OUT, SL.N_HID)
