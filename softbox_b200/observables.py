"""Per-network observables of device networks: RMS extent and contraction rate, largest-
cluster fraction, mean network stress.

    obs = Observables(net)                 # DenseNetwork, TurnoverNetwork or BatchedNetworks
    s = obs.sample()                        # {"rms_um", "rods", "largest", "active", "stress_pa"} per network
    rate = contraction_rate(times_s, rms_series)

Definitions (the reference has only the first, as a host diagnostic):
* R_rms: RMS distance of the ACTIVE filament rods' centres from their mean
  (FullSystemDemoHarness.filRms, FullSystemDemoHarness.java:1047-1055); the contraction
  rate is -d ln R_rms / dt, the least-squares slope over a time series;
* largest-cluster fraction: rods in the largest component / ACTIVE rods, components over
  rods and minifilament backbones joined by chain links, ACTIVE crosslinks and bound heads;
* mean stress: -(1/2V) sum (r_x F_x + r_y F_y) over the crosslink and cross-bridge force
  payloads of the last step (in-plane virial, Pa, positive = tension), V the slab volume.
All three run on the device (sbx_obs_*); a sample reads back a few numbers per network.
"""
import numpy as np

HEAD_LEN = 0.020                       # MotorStore.HEAD_LEN (um)


def motor_backbones(dim, mini, n_motors):
    """Backbone of every motor from the dimer tables (host arrays): -1 for a motor on no backbone."""
    mb = np.full(n_motors, -1, np.int32)
    hbs = np.asarray(mini["headBackboneSlot"])
    for key in ("motorA", "motorB"):
        m = np.asarray(dim[key])
        ok = m >= 0
        mb[m[ok]] = hbs[ok]
    return mb


def contraction_rate(times, rms):
    """-d ln R / dt by least squares (1/s)."""
    t = np.asarray(times, np.float64)
    y = np.log(np.asarray(rms, np.float64))
    tc = t - t.mean()
    return -float((tc * (y - y.mean())).sum() / (tc * tc).sum())


class Observables:
    def __init__(self, net, rounds=64):
        import torch
        d = net.dev
        self.dev, self.rounds = d, rounds
        info = getattr(net, "info", None)
        host = {k: {kk: vv for kk, vv in v.items() if kk in ("motorA", "motorB", "headBackboneSlot")}
                for k, v in (("dim", d["dim"]), ("mini", d["mini"]))}
        host = {k: {kk: vv.cpu().numpy() for kk, vv in v.items()} for k, v in host.items()}
        nS, nM = int(d["fil"]["body"]["n"]), int(d["mot"]["nMotors"])
        nL, nBb = int(d["xl"]["nLinks"]), int(d["mini"]["nBackbones"])
        i32 = dict(dtype=torch.int32, device=d["fil"]["filState"].device)
        if info is None:
            seg, link, mot = [0, nS], [0, nL], [0, nM]
            box = [d["boxParams"].cpu().numpy()]
        else:
            seg, link, mot = info["seg"], info["link"], info["mot"]
            box = d["batch"]["boxParams"].cpu().numpy().reshape(-1, 8)
        self.nNet = len(seg) - 1
        self.segBase = torch.tensor(np.asarray(seg, np.int32), **i32)
        self.linkBase = torch.tensor(np.asarray(link, np.int32), **i32)
        self.motBase = torch.tensor(np.asarray(mot, np.int32), **i32)
        self.volume = torch.tensor(np.array([b[1] * b[2] * b[3] for b in box], np.float32), dtype=torch.float32,
                                   device=self.segBase.device)
        self.motorBackbone = torch.tensor(motor_backbones(host["dim"], host["mini"], nM), **i32)
        self.nS, self.nM, self.nL, self.nBb = nS, nM, nL, nBb
        f64 = dict(dtype=torch.float64, device=self.segBase.device)
        self.ext = torch.zeros(2 * self.nNet, **f64)
        self.stress_out = torch.zeros(self.nNet, **f64)
        self.label = torch.zeros(nS + nBb, **i32)
        self.size = torch.zeros(nS + nBb, **i32)
        self.flags = torch.zeros(rounds + 1, **i32)
        self.cl = torch.zeros(2 * self.nNet, **i32)

    def _ctx(self):
        from .runtime import default_context
        return default_context()

    def extent(self):
        fb = self.dev["fil"]["body"]
        self._ctx()("sbx_obs_extent", self.nNet, self.segBase, self.nS, fb["coord"], fb.get("coord64"),
                    self.dev["fil"]["filState"], self.ext)
        return self.ext

    def stress(self):
        d = self.dev
        fb, xl, mot = d["fil"]["body"], d["xl"], d["mot"]
        self._ctx()("sbx_obs_stress", self.nNet, self.nS, fb["coord"], fb["uVec"], fb["end1"], fb["segLength"],
                    self.linkBase if self.nL else None, xl["linkFilA"], xl["linkFilB"], xl["linkState"], xl["loc1"],
                    xl["loc2"], xl["xlinkData"], self.nM, self.motBase if self.nM else None, mot["body"]["coord"],
                    mot["body"]["uVec"], mot["boundSeg"], mot["bindArc"], d["bondData"], HEAD_LEN, self.volume,
                    self.stress_out)
        return self.stress_out

    def clusters(self):
        d = self.dev
        xl, mot = d["xl"], d["mot"]
        self._ctx()("sbx_obs_clusters", self.nNet, self.segBase, self.nS, d["fil"]["filState"],
                    d["fil"]["end2NbrSlot"], self.nL, xl["linkFilA"], xl["linkFilB"], xl["linkState"], self.nM,
                    mot["boundSeg"], self.motorBackbone, self.nBb, self.rounds, self.label, self.size, self.flags,
                    self.cl)
        return self.cl

    def sample(self):
        """All three observables for every network (synchronises)."""
        self.extent()
        self.stress()
        self.clusters()
        ext = self.ext.cpu().numpy().reshape(-1, 2)
        cl = self.cl.cpu().numpy().reshape(-1, 2)
        if int(self.flags[self.rounds - 1].item()) != 0:
            raise RuntimeError("cluster labelling did not converge; raise `rounds`")
        return {"rms_um": ext[:, 0], "rods": ext[:, 1], "largest": cl[:, 0], "active": cl[:, 1],
                "largest_fraction": cl[:, 0] / np.maximum(cl[:, 1], 1), "stress_pa": self.stress_out.cpu().numpy()}
