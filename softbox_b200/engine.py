"""Device-resident networks: the public Python API over the fused step plans.

    net = DenseNetwork(scenes.dense_contractile(scenes.C1))
    net.run(t0=0, nsteps=100)          # "auto": one fused launch up to 40,960 rods, CUDA graphs above
    pose = net.pull("fil", "coord", sub="body")    # UNDER_DEMAND host copy

    rods = FreeRods(scenes.free_rods_box())
    rods.run(0, 10000, noise="wang")   # one persistent launch, rods in registers
"""
import ctypes as C

from . import device as D
from .runtime import LIB, SbxError, default_context


class DenseNetwork:
    """A dense contractile network (DenseContractileHarness.Scene) living on the device."""

    def __init__(self, host_scene, ctx=None, fp64_coords=False, device="cuda"):
        self.ctx = ctx or default_context()
        self.host = host_scene
        self.dev = D.to_device({k: v for k, v in host_scene.items() if k not in ("cfg", "tcfg")}, device)
        # motor, backbone and filament counts side by side: [nMotors, t, seed, nSeg,
        # nBackbones, t, seedBb, nBackbones, nSeg, t, seedFil, 1]
        self.counts_block = D.counts_block(self.dev)
        if fp64_coords:
            for path in (("fil", "body"), ("mot", "body"), ("mini", "backbone")):
                D.add_coord64(self.dev[path[0]][path[1]])
        self.desc = D.dense_desc(self.dev)
        self.plan = C.c_void_p()
        st = LIB.sbx_dense_plan_create(self.ctx.h, C.byref(self.desc), C.byref(self.plan))
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_create: " + self.ctx.last_error())

    MODES = {"unfused": 0, "graph": 1, "fused": 2, "auto": 3}

    @property
    def kernels_per_step(self):
        """Kernels one step launches on the graph path (the fused path launches one kernel per run)."""
        return LIB.sbx_dense_plan_kernels_per_step(self.plan)

    @property
    def fused_available(self):
        return bool(LIB.sbx_dense_plan_fused_available(self.plan))

    @property
    def fused_grid(self):
        return LIB.sbx_dense_plan_fused_grid(self.plan)

    def run(self, t0, nsteps, mode=None):
        """Advance steps t0..t0+nsteps-1. mode: "auto" (default: the fused kernel for
        networks up to SBX_DENSE_AUTO_MAX_FUSED_RODS rods when available, else the graph
        path), "fused" (one persistent cooperative launch for all steps), "graph" (one
        CUDA-graph replay per step) or "unfused" (the per-system call sequence). All give
        the same bits."""
        if mode is None:
            mode = "auto"
        st = LIB.sbx_dense_plan_run(self.plan, int(t0), int(nsteps), self.MODES[mode])
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_run: " + self.ctx.last_error())

    def status(self):
        """Synchronise and return the fused path's flags; raises on a timeout/overflow."""
        flags = C.c_int32(0)
        st = LIB.sbx_dense_plan_status(self.plan, C.byref(flags))
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_status: " + self.ctx.last_error())
        return flags.value

    def step_unfused(self, t):
        self.ctx("sbx_dense_step_unfused", self.desc, int(t))

    def set_noise(self, fil, mot, bb, t0):
        """Supplied-noise mode: steps t0 .. t0 + len(fil) - 1 take their Gaussians from the
        device arrays fil [nsteps][6][nRods], mot [nsteps][6][3 nMotors] and
        bb [nsteps][6][nBackbones] (float32, contiguous) instead of the Wang-hash draws.
        None switches the mode off. The arrays are kept alive by the network while in use."""
        from .abi_types import DenseNoiseDesc, _ptr
        if fil is None:
            self._noise = None
            st = LIB.sbx_dense_plan_set_noise(self.plan, None)
        else:
            nsteps = int(fil.shape[0])
            for x in (mot, bb):
                if int(x.shape[0]) != nsteps:
                    raise ValueError("noise arrays cover different step counts")
            d = DenseNoiseDesc()
            d.fil, d.mot, d.bb = _ptr(fil, C.c_float), _ptr(mot, C.c_float), _ptr(bb, C.c_float)
            d.t0, d.nsteps = int(t0), nsteps
            self._noise = (fil, mot, bb, d)
            st = LIB.sbx_dense_plan_set_noise(self.plan, C.byref(d))
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_set_noise: " + self.ctx.last_error())

    def fused_stats(self, reset=False):
        """The fused kernel's capacity-fallback counters (SBX_FUSED_STATS): cell overflow
        lists, link-end lists, motor lists, link payloads read past staging, motor reactions
        read past staging, motor rows walked by repeated minimum, reach lists past MAX_CAND."""
        out = (C.c_int64 * 8)()
        st = LIB.sbx_dense_plan_fused_stats(self.plan, out, 1 if reset else 0)
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_fused_stats: " + self.ctx.last_error())
        keys = ("cell_list", "link_list", "motor_list", "link_payload_global", "motor_payload_global",
                "motor_row_walk", "reach_over_cap")
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def test_caps(self, ent=-1, motor=-1, motor_ids=-1, row_slots=-1, cell_slots=-1):
        """Test hook: lowers the fused kernel's capacities (negative restores)."""
        st = LIB.sbx_dense_plan_test_caps(self.plan, int(ent), int(motor), int(motor_ids), int(row_slots),
                                          int(cell_slots))
        if st != 0:
            raise SbxError(st, "sbx_dense_plan_test_caps")

    def pull(self, store, field=None, sub=None):
        x = self.dev[store]
        if sub is not None:
            x = x[sub]
        if field is not None:
            x = x[field]
        return D.to_host(x)

    def pull_all(self):
        """Every device array of the network, copied to host (UNDER_DEMAND for all stores)."""
        return D.to_host(self.dev)

    def close(self):
        if self.plan:
            LIB.sbx_dense_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TurnoverNetwork(DenseNetwork):
    """A dense network with actin turnover (scenes.dense_turnover): at every biochem cadence
    the turnover block (growth, depolymerisation, death, severing, splits), the release of
    links and heads on dead slots, and constant-actin births run before that step's
    mechanics, all on the library's stream. The mechanics run on any path; on the fused
    path (mode "fused", or "auto" below the fused size limit) the plan re-reads the chain
    topology after each cadence (sbx_dense_plan_refresh: one stream synchronisation per
    cadence), since splits and births into FREE slots change the rod groups."""

    def __init__(self, host_scene, ctx=None, fp64_coords=False, device="cuda"):
        from .turnover import Turnover
        super().__init__(host_scene, ctx=ctx, fp64_coords=fp64_coords, device=device)
        d = self.dev
        self.tcfg = host_scene["tcfg"]
        xl = d["xl"]
        self.turnover = Turnover(d["fil"], d["turnover"], self.tcfg,
                                 links=(xl["linkFilA"], xl["linkFilB"], xl["linkState"]),
                                 boundSeg=d["mot"]["boundSeg"])

    def run(self, t0, nsteps, mode="auto"):
        if mode not in self.MODES:
            raise ValueError(f"unknown mode {mode!r}")
        t, end = int(t0), int(t0) + int(nsteps)
        ci = self.tcfg.check_int
        while t < end:
            if self.tcfg.fires_at(t):
                self.turnover.cadence(t)
                self.turnover.births(t)
                if mode in ("fused", "auto"):
                    st = LIB.sbx_dense_plan_refresh(self.plan)
                    if st != 0:
                        raise SbxError(st, "sbx_dense_plan_refresh: " + self.ctx.last_error())
            nxt = min(end, (t // ci + 1) * ci)
            super().run(t, nxt - t, mode)
            t = nxt


class FreeRods:
    """Free Brownian rods (DiffusionHarness Config T/R and the free-rod workload)."""

    MODES = {"wang": 0, "philox": 1, "supplied": 2}

    def __init__(self, host_store, ctx=None, fp64_coords=False, device="cuda"):
        self.ctx = ctx or default_context()
        self.dev = D.to_device(host_store, device)
        if fp64_coords:
            D.add_coord64(self.dev["body"])
        self.desc = D.filament_desc(self.dev)

    def run(self, t0, nsteps, noise="wang", philox_seed=0, supplied=None):
        self.ctx("sbx_free_rods_run", self.desc, int(t0), int(nsteps), self.MODES[noise], int(philox_seed), supplied)

    def pull(self, field):
        return D.to_host(self.dev["body"][field])
