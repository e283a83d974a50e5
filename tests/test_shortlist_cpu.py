"""The shortlist network's CPU restatement (the checker of its GPU training kernels): bf16 rounding, im2col / col2im
as adjoints, and analytic gradients against finite differences; the initial parameters are seeded."""
import numpy as np

import shortlist_ref as R
from av1gpu_b200 import shortlist as SL


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, -3.14159, 65504.0, 1e-30], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0078125 or r[1] == 1.0   # halfway cases go to even
    assert abs(r[3] - (-3.140625)) < 1e-9
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8 + 1e-38)


def test_layout_matches_the_library():
    assert R.N_PARAMS == SL.N_PARAMS == 62688
    assert [s for _, s in R.SHAPES] == [s for _, s in SL.SHAPES]
    # the (mode, delta) classes: 5 non-directional modes at delta 0, then V .. D67 x delta -3 .. 3
    assert len(set(SL.CLASS_CAND.tolist())) == 61
    assert [c >> 3 for c in SL.CLASS_CAND[:5]] == [0, 9, 10, 11, 12] and all((c & 7) == 3 for c in SL.CLASS_CAND[:5])
    assert SL.CLASS_CAND[5] == (1 << 3 | 0) and SL.CLASS_CAND[60] == (8 << 3 | 6)


def test_im2col_col2im_adjoint():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((3, 8, 8, 5))
    d = rng.standard_normal((3 * 16, 45))
    assert abs(float((R.im2col(x) * d).sum()) - float((x * R.col2im(d, 3, 8, 8, 5)).sum())) < 1e-9
    # tap 4 is the centre: column block 4 of im2col is the stride-2 subsample
    assert np.array_equal(R.im2col(x)[:, 4 * 5:5 * 5].reshape(3, 4, 4, 5), x[:, ::2, ::2, :])


def _rows(rng, n):
    X = rng.standard_normal((n, R.N_FEAT)) * 0.5
    y = np.zeros((n, 3), np.int64)
    y[:, 0] = rng.integers(0, R.N_MD, n)
    sets = np.array([0b111000001111, 0b1000001111, 0])   # INTRA_1 (7 types), INTRA_2 (5), DCT_DCT alone
    for r in range(n):
        v = int(sets[r % 3])
        y[r, 2] = v
        ks = [k for k in range(16) if (v >> k) & 1]
        y[r, 1] = rng.choice(ks) if ks else -1
    return X, y


def test_restated_gradients_by_finite_differences():
    rng = np.random.default_rng(0)
    n = 6
    X, y = _rows(rng, n)
    p = SL.init_params(2).astype(np.float64)
    p[R.N_PARAMS - 80:] += rng.standard_normal(80) * 0.1   # fc2 biases
    ident = lambda a: np.asarray(a, np.float64)  # noqa: E731
    g, loss, _ = R.grads(X, y, p, rnd=ident)

    def L(q):
        return R.loss_grad_scores(R.forward(X, q, rnd=ident)["s"], y)[0]
    assert abs(loss - L(p)) < 1e-12
    eps = 1e-6
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in R.SHAPES])
    for k in range(len(R.SHAPES)):   # a few entries of every parameter array
        for i in rng.integers(offs[k], offs[k + 1], 3):
            q = p.copy()
            q[i] += eps
            lp = L(q)
            q[i] -= 2 * eps
            lm = L(q)
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[i]) < 1e-6 + 1e-4 * abs(num), (R.SHAPES[k][0], i, num, g[i])


def test_init_params_seeded():
    a, b = SL.init_params(7), SL.init_params(7)
    assert np.array_equal(a, b) and a.dtype == np.float32 and a.size == SL.N_PARAMS
    assert not np.array_equal(a, SL.init_params(8))
