"""The surrogate ensemble on the GPU: forward outputs and every gradient of one training
step against the CPU oracle (same BF16 weights and inputs), then training that fits a
smooth function of the six inputs better than the mean predictor."""
import numpy as np
import pytest

import mlp_oracle as mo

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bits_to_f32(t):
    return mo.from_bits(t.cpu().numpy().view(np.uint16))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_and_gradients_match_oracle():
    from softbox_b200.surrogate import MLPEnsemble
    ens = MLPEnsemble(n_nets=3, batch=256, seed=4)
    rng = np.random.default_rng(7)
    x = torch.tensor(rng.normal(size=(3, 256, 6)), dtype=torch.float32, device="cuda")
    y = torch.tensor(rng.normal(size=(3, 256, 3)), dtype=torch.float32, device="cuda")
    ens._stage_inputs(x)
    ens.T.copy_(y)
    ens.forward()
    ens.backward()
    torch.cuda.synchronize()
    assert ens.err.item() == 0
    X0 = _bits_to_f32(ens.X0).reshape(3, 256, 16)
    for z in range(3):
        W = [_bits_to_f32(ens.Wb[l]).reshape(ens.nz, ens.Np[l], ens.Kp[l])[z] for l in range(ens.L)]
        b = [ens.b[l].cpu().numpy()[z] for l in range(ens.L)]
        Z, A = mo.forward(X0[z], W, b)
        out = ens.Z[-1].cpu().numpy()[z]
        assert _rel(out[:, :3], Z[-1][:, :3]) < 1e-2
        assert np.abs(out[:, 3:]).max() == 0                      # padded outputs stay zero
        dW, db, loss = mo.backward(Z, A, W, y.cpu().numpy()[z], 3)
        for l in range(ens.L):
            g = ens.dW[l].cpu().numpy()[z]
            assert _rel(g, dW[l]) < 2e-2, f"dW layer {l}"
            assert _rel(ens.db[l].cpu().numpy()[z], db[l]) < 2e-2, f"db layer {l}"
        assert abs(ens.loss.cpu().numpy()[z] - loss) < 1e-3 * loss
        assert np.abs(ens.dW[0].cpu().numpy()[z][:, 6:]).max() == 0   # padded inputs get no gradient
        assert np.abs(ens.dW[-1].cpu().numpy()[z][3:]).max() == 0     # padded outputs neither


def test_training_fits_a_smooth_target():
    from softbox_b200.surrogate import MLPEnsemble, fallback_mask
    rng = np.random.default_rng(1)
    X = rng.uniform(size=(4096, 6))
    Y = np.stack([np.sin(3 * X[:, 0]) + X[:, 1] * X[:, 2], np.exp(-X[:, 3]) * 2 + 1, X[:, 4] - X[:, 5] ** 2 + 2],
                 axis=1)
    ens = MLPEnsemble(n_nets=5, seed=2)
    hist = ens.fit(X[:3584], Y[:3584], epochs=30)
    assert hist[-1] < 0.05 * hist[0]
    mean, std, _ = ens.predict(X[3584:])
    err = np.abs(mean - Y[3584:]) / np.abs(Y[3584:]).mean(axis=0)
    assert err.mean() < 0.05
    assert fallback_mask(mean, std, 0.10).mean() < 0.5
