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


@pytest.mark.parametrize("ldo_pad", [0, 3], ids=["vector-rows", "scalar-rows"])
def test_gemm_epilogue_matches_torch(ldo_pad):
    """sbx_mlp_gemm_bf16 on ragged sizes (M, N and K not multiples of the tiles), two problems
    in one launch, with bias + GELU and all three outputs, against torch on the same BF16
    operands: the FP32 pre-activations to FP32 accumulation-order tolerance, the BF16
    activations and their transpose to one BF16 rounding. ldo_pad > 0 makes the row-major
    outputs' rows unaligned (the element-wise store path)."""
    from softbox_b200.runtime import Context
    nz, M, N, K = 2, 1000, 200, 100
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(nz, M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (0.1 * torch.randn(nz, N, K, device="cuda", generator=g)).to(torch.bfloat16)
    bias = torch.randn(nz, N, device="cuda", generator=g)
    ldo = N + ldo_pad
    out = torch.zeros(nz, M, ldo, dtype=torch.bfloat16, device="cuda")
    outF = torch.zeros(nz, M, ldo, dtype=torch.float32, device="cuda")
    outT = torch.zeros(nz, N, M, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ctx = Context(0)
    ctx("sbx_mlp_gemm_bf16", nz, M, N, K, A, K, M * K, B, K, N * K, bias, N, 1, out, ldo, M * ldo, outT, M, N * M,
        outF, ldo, M * ldo, err)
    ctx.sync()
    assert err.item() == 0
    v = torch.matmul(A.float(), B.float().transpose(1, 2)) + bias[:, None, :]
    a = torch.nn.functional.gelu(v)
    got_v = outF[:, :, :N]
    assert torch.allclose(got_v, v, rtol=1e-4, atol=1e-4), (got_v - v).abs().max()
    ref = a.to(torch.bfloat16).float()
    for got in (out[:, :, :N].float(), outT.transpose(1, 2).float()):
        # one BF16 rounding of values that agree to FP32 accumulation order
        assert torch.allclose(got, ref, rtol=1e-2, atol=1e-2), (got - ref).abs().max()
    # padding columns of the row-major outputs stay untouched
    if ldo_pad:
        assert out[:, :, N:].float().abs().max().item() == 0
        assert outF[:, :, N:].abs().max().item() == 0
