"""The tensor-core BF16 GEMM against the oracle: shapes with partial tiles, padding of K
and N, bias, GELU, FP32 / BF16 / transposed outputs, several ensemble members."""
import numpy as np
import pytest

import mlp_oracle as mo

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev_bf16(x):
    return torch.from_numpy(mo.bf16_bits(x).view(np.int16)).cuda()


def _host_bf16(t):
    return mo.from_bits(t.cpu().numpy().view(np.uint16))


@pytest.mark.parametrize("M,N,K,act", [(256, 256, 256, 1), (300, 200, 100, 0), (128, 16, 6, 1), (77, 256, 16, 0),
                                       (1000, 48, 256, 1)])
def test_gemm_matches_oracle(M, N, K, act):
    from softbox_b200.systems import _ctx
    nz = 3
    rng = np.random.default_rng(M + N + K)
    A = mo.bf16(rng.normal(size=(nz, M, K)).astype(np.float32))
    B = mo.bf16((rng.normal(size=(nz, N, K)) / np.sqrt(K)).astype(np.float32))
    bias = rng.normal(size=(nz, N)).astype(np.float32)
    dA, dB = _dev_bf16(A), _dev_bf16(B)
    db = torch.from_numpy(bias).cuda()
    out = torch.zeros((nz, M, N), dtype=torch.int16, device="cuda")
    outT = torch.zeros((nz, N, M), dtype=torch.int16, device="cuda")
    outF = torch.zeros((nz, M, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _ctx()("sbx_mlp_gemm_bf16", nz, M, N, K, dA, K, M * K, dB, K, N * K, db, N, act, out, N, M * N, outT, M, N * M,
           outF, N, M * N, err)
    torch.cuda.synchronize()
    assert err.item() == 0
    f = outF.cpu().numpy()
    o = _host_bf16(out).reshape(nz, M, N)
    ot = _host_bf16(outT).reshape(nz, N, M)
    for z in range(nz):
        Z, Ab = mo.gemm(A[z], B[z], bias[z], act=bool(act))
        scale = np.abs(Z).max()
        assert np.abs(f[z] - Z).max() <= 1e-5 * scale, "FP32 accumulation"
        # BF16 outputs: the same rounding except where the FP32 sum sits at a rounding boundary
        assert np.abs(o[z] - Ab).max() <= 2 ** -7 * max(1.0, np.abs(Ab).max())
        assert (o[z] != Ab).mean() < 0.01
        assert np.array_equal(ot[z], o[z].T)
