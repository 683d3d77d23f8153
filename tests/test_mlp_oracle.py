"""The MLP oracle itself (CPU): its backward pass against central finite differences of its
own loss with the BF16 rounding switched off, and the BF16 rounding helper."""
import numpy as np

import mlp_oracle as mo


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39, 65504.0], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie (1 + 2^-8) rounds to even
    assert r[2] == np.float32(1.0078125)          # above the tie rounds up
    assert r[3] == -2.5
    assert np.array_equal(mo.from_bits(mo.bf16_bits(x)), r)


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(mo, "rnd", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(0)
    dims = [6, 12, 12, 3]
    W = [rng.normal(size=(dims[i + 1], dims[i])) / np.sqrt(dims[i]) for i in range(3)]
    b = [rng.normal(size=dims[i + 1]) * 0.1 for i in range(3)]
    x = rng.normal(size=(9, 6))
    t = rng.normal(size=(9, 3))
    Z, A = mo.forward(x, W, b)
    dW, db, loss = mo.backward(Z, A, W, t, 3)

    def loss_of(W_, b_):
        Z_, _ = mo.forward(x, W_, b_)
        return float(((Z_[-1][:, :3] - t) ** 2).mean())

    h = 1e-6
    for l in range(3):
        for (i, j) in ((0, 0), (1, 2), (dims[l + 1] - 1, dims[l] - 1)):
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[l][i, j] += h
            Wm[l][i, j] -= h
            fd = (loss_of(Wp, b) - loss_of(Wm, b)) / (2 * h)
            assert abs(fd - dW[l][i, j]) <= 1e-6 * max(1.0, abs(fd))
        bp = [v.copy() for v in b]
        bm = [v.copy() for v in b]
        bp[l][1] += h
        bm[l][1] -= h
        fd = (loss_of(W, bp) - loss_of(W, bm)) / (2 * h)
        assert abs(fd - db[l][1]) <= 1e-6 * max(1.0, abs(fd))
