"""Surrogate of the parameter sweep: an ensemble of MLPs trained and evaluated on the
device by the library's tensor-core kernels (sbx_mlp_*), with the plain simulation as the
fallback wherever the ensemble disagrees.

    ens = MLPEnsemble()                             # 5 nets, 6 -> 256 x4 (GELU) -> 3, BF16
    ens.fit(X, Y, epochs=...)                        # Adam, lr 1e-3, batch 256
    mean, std = ens.predict(X_new)                   # per output, de-normalised
    rerun = fallback_mask(mean, std, 0.10)           # points for the plain simulator

Every GEMM of the forward and backward passes (C = A B^T with BF16 operands and FP32
accumulation in tensor memory) is sbx_mlp_gemm_bf16 with all ensemble members in one
launch (blockIdx.z); the epilogues write the BF16 activations, their transposes (the
operands of the weight-gradient GEMMs) and the FP32 pre-activations. The GELU backward,
bias gradients, loss gradient and Adam (FP32 master weights, BF16 copies and transposes)
are the library's elementwise kernels. Torch provides the device buffers and the batch
gathers only.

Shapes are padded for the tensor cores: the 6 inputs to 16 columns and the 3 outputs to
16 rows of the last weight matrix; the padding stays exactly zero (zero inputs and zero
output gradients give it zero gradients).
"""
import numpy as np

KPAD_IN = 16
NPAD_OUT = 16


class MLPEnsemble:
    def __init__(self, n_nets=5, dims=(6, 256, 256, 256, 256, 3), batch=256, seed=0, lr=1e-3, device="cuda"):
        import torch
        self.torch = torch
        self.nz, self.dims, self.B, self.lr = n_nets, tuple(dims), batch, lr
        self.L = len(dims) - 1
        self.nin, self.nout = dims[0], dims[-1]
        self.Kp = [KPAD_IN] + [dims[l] for l in range(1, self.L)]
        self.Np = [dims[l + 1] for l in range(self.L - 1)] + [NPAD_OUT]
        self.dev = device
        self.step_no = 0
        rng = np.random.default_rng(seed)
        f32 = dict(dtype=torch.float32, device=device)
        i16 = dict(dtype=torch.int16, device=device)
        self.W, self.Wb, self.WbT, self.b = [], [], [], []
        self.mW, self.vW, self.mb, self.vb, self.dW, self.db = [], [], [], [], [], []
        for l in range(self.L):
            fin, fout = dims[l], dims[l + 1]
            w = np.zeros((n_nets, self.Np[l], self.Kp[l]), np.float32)
            w[:, :fout, :fin] = rng.uniform(-1, 1, (n_nets, fout, fin)) * np.sqrt(3.0 / fin)
            bb = np.zeros((n_nets, self.Np[l]), np.float32)
            self.W.append(torch.from_numpy(w).to(device))
            self.b.append(torch.from_numpy(bb).to(device))
            self.Wb.append(torch.zeros((n_nets, self.Np[l], self.Kp[l]), **i16))
            self.WbT.append(torch.zeros((n_nets, self.Kp[l], self.Np[l]), **i16))
            for lst in (self.mW, self.vW, self.dW):
                lst.append(torch.zeros((n_nets, self.Np[l], self.Kp[l]), **f32))
            for lst in (self.mb, self.vb, self.db):
                lst.append(torch.zeros((n_nets, self.Np[l]), **f32))
        self._refresh_bf16()
        self._alloc(batch)
        self.x_mean = self.x_std = self.y_mean = self.y_std = None
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.graph = None

    # ---------------------------------------------------------------- buffers
    def _alloc(self, M):
        t = self.torch
        f32 = dict(dtype=t.float32, device=self.dev)
        i16 = dict(dtype=t.int16, device=self.dev)
        nz = self.nz
        self.M = M
        self.X0 = t.zeros((nz, M, KPAD_IN), **i16)
        self.X0T = t.zeros((nz, KPAD_IN, M), **i16)
        self.T = t.zeros((nz, M, self.nout), **f32)
        self.Z = [t.zeros((nz, M, self.Np[l]), **f32) for l in range(self.L)]
        self.A = [t.zeros((nz, M, self.Np[l]), **i16) for l in range(self.L)]
        self.AT = [t.zeros((nz, self.Np[l], M), **i16) for l in range(self.L)]
        self.G = [t.zeros((nz, M, self.Np[l]), **i16) for l in range(self.L)]
        self.GT = [t.zeros((nz, self.Np[l], M), **i16) for l in range(self.L)]
        self.dA = [t.zeros((nz, M, self.Kp[l]), **f32) for l in range(self.L)]     # dL / d(input of layer l)
        self.gout = t.zeros((nz, M, NPAD_OUT), **f32)
        self.loss = t.zeros(nz, **f32)

    def _ctx(self):
        from .runtime import default_context
        return default_context()

    def _refresh_bf16(self):
        """BF16 copies (and transposes) of the FP32 master weights (at initialisation)."""
        t = self.torch
        for l in range(self.L):
            wb = self.W[l].to(t.bfloat16)
            self.Wb[l].copy_(wb.view(t.int16))
            self.WbT[l].copy_(wb.transpose(1, 2).contiguous().view(t.int16))

    # ---------------------------------------------------------------- passes
    def _gemm(self, M, N, K, A, lda, sA, B, ldb, sB, bias=None, act=0, out=None, outT=None, outF=None, ldt=None):
        ctx = self._ctx()
        ctx("sbx_mlp_gemm_bf16", self.nz, M, N, K, A, lda, sA, B, ldb, sB, bias, 0 if bias is None else bias.shape[-1],
            act, out, N, 0 if out is None else out[0].numel(), outT, ldt or M, 0 if outT is None else outT[0].numel(),
            outF, N, 0 if outF is None else outF[0].numel(), self.err)

    def forward(self, M=None, keep_t=True):
        """Forward pass over the staged inputs X0 (M rows); keep_t=False (inference) writes
        only the activations and the last layer's output."""
        M = M or self.M
        prev, lda = self.X0, KPAD_IN
        for l in range(self.L):
            last = l == self.L - 1
            self._gemm(M, self.Np[l], self.Kp[l], prev, lda, prev[0].numel(), self.Wb[l], self.Kp[l],
                       self.Wb[l][0].numel(), bias=self.b[l], act=0 if last else 1, out=None if last else self.A[l],
                       outT=self.AT[l] if (keep_t and not last) else None,
                       outF=self.Z[l] if (keep_t or last) else None)
            prev, lda = self.A[l], self.Np[l]
        return self.Z[-1]

    def backward(self):
        ctx = self._ctx()
        M, nz = self.M, self.nz
        self.loss.zero_()
        ctx("sbx_mlp_mse_grad", nz, M, NPAD_OUT, self.nout, self.Z[-1], self.Z[-1][0].numel(), self.T,
            self.T[0].numel(), self.gout, self.gout[0].numel(), self.loss)
        ctx("sbx_mlp_gelu_backward", nz, M, NPAD_OUT, self.gout, None, self.gout[0].numel(), self.G[-1], self.GT[-1],
            self.G[-1][0].numel(), self.GT[-1][0].numel())
        for l in range(self.L - 1, -1, -1):
            N, K = self.Np[l], self.Kp[l]
            ctx("sbx_mlp_colsum_bf16", nz, M, N, self.G[l], self.G[l][0].numel(), self.db[l], N)
            # dW_l = G_l^T . A_{l-1}: C[N x K] = GT[N x M] . (A_{l-1}^T)[K x M]^T
            AprevT = self.X0T if l == 0 else self.AT[l - 1]
            self._gemm(N, K, M, self.GT[l], M, self.GT[l][0].numel(), AprevT, M, AprevT[0].numel(),
                       outF=self.dW[l])
            if l > 0:
                # dA_{l-1} = G_l . W_l: C[M x K] = G[M x N] . (W_l^T)[K x N]^T
                self._gemm(M, K, N, self.G[l], N, self.G[l][0].numel(), self.WbT[l], N, self.WbT[l][0].numel(),
                           outF=self.dA[l])
                ctx("sbx_mlp_gelu_backward", nz, M, K, self.dA[l], self.Z[l - 1], self.Z[l - 1][0].numel(),
                    self.G[l - 1], self.GT[l - 1], self.G[l - 1][0].numel(), self.GT[l - 1][0].numel())

    def adam(self):
        ctx = self._ctx()
        self.step_no += 1
        for l in range(self.L):
            N, K = self.Np[l], self.Kp[l]
            ctx("sbx_mlp_adam", self.nz, N, K, self.W[l], self.dW[l], self.mW[l], self.vW[l], N * K, self.lr, 0.9,
                0.999, 1e-8, self.step_no, self.Wb[l], self.WbT[l], N * K, N * K)
            ctx("sbx_mlp_adam", self.nz, N, 1, self.b[l], self.db[l], self.mb[l], self.vb[l], N, self.lr, 0.9, 0.999,
                1e-8, self.step_no, None, None, 0, 0)

    # ---------------------------------------------------------------- data
    def _stage_inputs(self, x):
        """x: [nz, M, nin] float tensor (normalised) -> X0 and X0T (BF16, padded to 16)."""
        t = self.torch
        nz, M = x.shape[0], x.shape[1]
        xp = t.zeros((nz, M, KPAD_IN), dtype=t.bfloat16, device=self.dev)
        xp[:, :, :self.nin] = x.to(t.bfloat16)
        self.X0[:, :M].copy_(xp.view(t.int16))
        self.X0T[:, :, :M].copy_(xp.transpose(1, 2).contiguous().view(t.int16))

    def set_normalisation(self, X, Y):
        X = np.asarray(X, np.float64)
        Y = np.asarray(Y, np.float64)
        self.x_mean, self.x_std = X.mean(0), X.std(0) + 1e-8
        self.y_mean, self.y_std = Y.mean(0), Y.std(0) + 1e-8

    def train_step(self, xb, tb):
        """One Adam step per member on its own batch: xb [nz, B, nin], tb [nz, B, nout]
        (normalised, device). Returns nothing; the losses stay in self.loss."""
        self._stage_inputs(xb)
        self.T.copy_(tb)
        self.forward()
        self.backward()
        self.adam()

    def fit(self, X, Y, epochs=100, seed=0, log=None, bootstrap=False):
        """Trains every member on (X, Y) with its own shuffling (with `bootstrap`, each member
        on its own resample of the points drawn with replacement, so the members' spread
        reflects what the data leaves open); returns the loss history."""
        t = self.torch
        if self.x_mean is None:
            self.set_normalisation(X, Y)
        Xn = t.tensor((np.asarray(X) - self.x_mean) / self.x_std, dtype=t.float32, device=self.dev)
        Yn = t.tensor((np.asarray(Y) - self.y_mean) / self.y_std, dtype=t.float32, device=self.dev)
        n = Xn.shape[0]
        g = t.Generator(device="cpu").manual_seed(seed)
        samples = [t.randint(0, n, (n,), generator=g) if bootstrap else t.arange(n) for _ in range(self.nz)]
        hist = []
        steps = max(1, n // self.B)
        for ep in range(epochs):
            perms = t.stack([smp[t.randperm(n, generator=g)] for smp in samples]).to(self.dev)
            for s in range(steps):
                idx = perms[:, s * self.B:(s + 1) * self.B]
                if idx.shape[1] < self.B:
                    break
                self.train_step(Xn[idx], Yn[idx])
            hist.append(float(self.loss.mean().item()))
            if log:
                log(ep, hist[-1])
        return hist

    def _alloc_infer(self, M):
        """Inference buffers for up to M points per chunk, kept between calls: the staged
        inputs, the hidden activations and the last layer's FP32 output (nothing of the
        training passes)."""
        t = self.torch
        nz = self.nz
        self._inf_M = M
        self._inf_X0 = t.zeros((nz, M, KPAD_IN), dtype=t.int16, device=self.dev)
        self._inf_A = [t.empty((nz, M, self.Np[l]), dtype=t.int16, device=self.dev) for l in range(self.L - 1)]
        self._inf_Z = t.empty((nz, M, self.Np[-1]), dtype=t.float32, device=self.dev)

    def _forward_infer(self, M):
        """The forward pass of the first M staged inference rows; returns the output buffer."""
        prev, lda = self._inf_X0, KPAD_IN
        for l in range(self.L):
            last = l == self.L - 1
            self._gemm(M, self.Np[l], self.Kp[l], prev, lda, prev[0].numel(), self.Wb[l], self.Kp[l],
                       self.Wb[l][0].numel(), bias=self.b[l], act=0 if last else 1,
                       out=None if last else self._inf_A[l], outF=self._inf_Z if last else None)
            if not last:
                prev, lda = self._inf_A[l], self.Np[l]
        return self._inf_Z

    def predict(self, X, chunk=65536):
        """Ensemble mean and standard deviation of the de-normalised outputs for X [P, nin].
        Runs on inference buffers of its own (allocated on first use of a chunk size, then
        reused), so a prediction allocates nothing once they exist."""
        t = self.torch
        Xn = t.tensor((np.asarray(X) - self.x_mean) / self.x_std, dtype=t.float32, device=self.dev)
        P = Xn.shape[0]
        need = min(max(P, 1), chunk)
        if getattr(self, "_inf_M", 0) < need:
            self._alloc_infer(need)
        outs = []
        for c0 in range(0, P, chunk):
            xc = Xn[c0:c0 + chunk]
            m = xc.shape[0]
            xp = t.zeros((m, KPAD_IN), dtype=t.bfloat16, device=self.dev)
            xp[:, :self.nin] = xc.to(t.bfloat16)
            self._inf_X0[:, :m].copy_(xp.view(t.int16).unsqueeze(0).expand(self.nz, m, KPAD_IN))
            outs.append(self._forward_infer(m)[:, :m, :self.nout].clone())
        y = t.cat(outs, dim=1).cpu().numpy().astype(np.float64) * self.y_std + self.y_mean
        return y.mean(axis=0), y.std(axis=0), y


def fallback_mask(mean, std, threshold=0.10, outputs=None, scale=None):
    """Points where an output's ensemble std exceeds `threshold` of its |mean| (any of the
    `outputs` columns, default all); with `scale` (one value per output) |mean| is floored at
    it, so outputs whose mean sits near zero do not fall back on their absolute noise alone."""
    ref = np.abs(mean)
    if scale is not None:
        ref = np.maximum(ref, np.asarray(scale)[None, :])
    over = std > threshold * ref
    if outputs is not None:
        over = over[:, list(outputs)]
    return over.any(axis=1)


def select_rule(mean_v, std_v, y_v, mean_f, std_f, spread, infer_s, rerun_s_per_point, per_run_s, target_col=0,
                max_err=0.05, thresholds=(0.05, 0.1, 0.2, 0.3, 0.5), floors=(0.0, 0.25, 0.5, 1.0),
                output_sets=((0, 1, 2), (0,))):
    """Picks the fallback rule (outputs checked, threshold, floor as a fraction of each output's
    training spread) with the highest sweep rate whose relative error on column `target_col`
    over the validation points (mean_v, std_v against plain runs y_v; fallback points take their
    plain result) stays within max_err. The sweep rate of a rule is len(mean_f) fresh points
    over inference time plus a plain rerun for each fresh fallback point; gain = rate x the
    plain per-run seconds. Returns (best rule or None, every rule's row)."""
    rows = []
    for outs in output_sets:
        for th in thresholds:
            for fl in floors:
                sc = fl * spread if fl > 0 else None
                fb_v = fallback_mask(mean_v, std_v, th, outs, sc)
                blend = np.where(fb_v[:, None], y_v, mean_v)
                err = np.abs(blend - y_v).mean(axis=0) / np.maximum(np.abs(y_v).mean(axis=0), 1e-30)
                fb_f = fallback_mask(mean_f, std_f, th, outs, sc)
                rate = len(mean_f) / (infer_s + int(fb_f.sum()) * rerun_s_per_point)
                rows.append({"outputs": list(outs), "threshold": th, "floor": fl,
                             "validation_fallback": float(fb_v.mean()), "validation_rel_error": err.tolist(),
                             "fresh_fallback": float(fb_f.mean()), "points_per_s": rate,
                             "gain_vs_plain_per_run": rate * per_run_s})
    ok = [r for r in rows if r["validation_rel_error"][target_col] <= max_err]
    best = max(ok, key=lambda r: r["points_per_s"]) if ok else None
    return best, rows


def main():
    """Times ensemble inference: python -m softbox_b200.surrogate [--points 100000] [--repeat 5]"""
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=100000)
    ap.add_argument("--repeat", type=int, default=5)
    a = ap.parse_args()
    rng = np.random.default_rng(0)
    x = rng.uniform(size=(a.points, 6))
    ens = MLPEnsemble()
    ens.set_normalisation(x, np.zeros((1, 3)))
    ens.predict(x)                                  # warm-up: the inference buffers exist after it
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(True), torch.cuda.Event(True)
    s.record()
    for _ in range(a.repeat):
        ens.predict(x)
    e.record()
    torch.cuda.synchronize()
    sec = s.elapsed_time(e) / 1e3 / a.repeat
    flops = 2.0 * a.points * ens.nz * sum(ens.Np[l] * ens.Kp[l] for l in range(ens.L))
    print(json.dumps({"points": a.points, "nets": ens.nz, "s_per_predict": sec, "points_per_s": a.points / sec,
                      "gemm_tflops_incl_host": flops / sec / 1e12}), flush=True)


if __name__ == "__main__":
    main()
