"""Host-side stores and scene builders.

Arrays follow the reference's planar SoA store layouts (FilamentStore.java:10-22:
[x0..xN-1 | y0..yN-1 | z0..zN-1]) and field names, so a scene built here is the same
data a reference harness would hand to its System classes. Builders restate the
reference harnesses' host set-up:

  * free_rods_fdt      DiffusionHarness.freshStore        (DiffusionHarness.java:742-755)
  * deflection_chain   DiffusionHarness.measureDeflection (DiffusionHarness.java:287-335)
  * free_rods_box      the free-Brownian-rod workload (1,024 rods of 1.0 um in a 10 um box)
  * dense_contractile  DenseContractileHarness.buildScene (DenseContractileHarness.java:112-280)
                       with the network composition as a parameter set (DenseConfig)

Host initialisation (drag tensors, Brownian amplitudes) runs here in double precision
exactly as the reference's host code does (DragTensorSystem.java:33-97).
"""
import math
from dataclasses import dataclass, field, replace

import numpy as np

from .javarandom import JavaRandom

F32 = np.float32
I32 = np.int32

# Constants.java:25-67
BOLTZ = 1.380662e-23
TEMP_K = 298.15
KT = BOLTZ * TEMP_K
ACTIN_MONO_RADIUS = 0.0054 / 2.0
ACTIN_RADIUS = 0.007 / 2.0
STD_SEG_LENGTH = 32
A_PARALLEL, A_ORTHOG, A_TURNING = -0.20, 0.84, -0.662
BTRANS_COEFF, BROT_COEFF = 1.0, 0.5
PERSISTENCE_LENGTH = 15.0
EI = KT * (PERSISTENCE_LENGTH * 1.0e-6)
# MotorStore.java:45-46, MiniFilamentStore.java:34-38, DimerStore.java:40-43
ROD_LEN, LEVER_LEN, HEAD_LEN = 0.080, 0.008, 0.020
ROD_R, LEVER_R, HEAD_R = 0.003, 0.002, 0.010
BACKBONE_R = 0.005
MINIFIL_FRAC_MOVE, MINIFIL_ALIGN = 0.07, 0.01
DIMER_ROD_FRAC_MOVE, DIMER_LEVER_FMT, DIMER_LEVER_DEG = 0.2, 0.4, 160.0
STORE_FILAMENT, STORE_MOTOR, STORE_NONE = 0, 1, -1
MAX_CAND = 256
GRID_SCAN_CHUNK = 512
XB_STRIDE, XL_STRIDE, MINI_STRIDE = 13, 12, 6
STRAIN_WIN, TORQUE_WIN = 10, 5
NUC_NONE, NUC_ATP, NUC_ADPPI, NUC_ADP = 0, 1, 2, 3
MYO_REBIND_TIME = 1.0e-5
SIN80 = math.sin(math.radians(80.0))
COS80 = math.cos(math.radians(80.0))


def rod_drag_si(length_um, radius_um, aeta):
    """DragTensorSystem.rodDragSI (DragTensorSystem.java:33-45)."""
    LM = 1.0e-6 * length_um
    RM = radius_um * 1.0e-6
    logT = math.log(LM / (2 * RM))
    bTGx = (2 * math.pi * aeta * LM) / (logT + A_PARALLEL)
    bTGy = (4 * math.pi * aeta * LM) / (logT + A_ORTHOG)
    bRGx = 4 * math.pi * aeta * RM * RM * LM
    bRGy = (math.pi * aeta * (LM * LM * LM)) / (3 * (logT + A_TURNING))
    return [bTGx, bTGy, bTGy, bRGx, bRGy, bRGy]


def sphere_drag_si(radius_um, aeta):
    """DragTensorSystem.sphereDragSI (DragTensorSystem.java:52-58)."""
    RM = radius_um * 1.0e-6
    bTG = 6 * math.pi * aeta * RM
    bRG = 8 * math.pi * aeta * (RM * RM * RM)
    return [bTG, bTG, bTG, bRG, bRG, bRG]


def rigid_body(n):
    """RigidRodBody.java:59-84 — all arrays zero."""
    b = {k: np.zeros(3 * n, F32) for k in ("coord", "uVec", "yVec", "zVec", "end1", "end2", "bTransGam",
                                           "bRotGam", "bTransDiff", "bRotDiff", "forceSum", "torqueSum",
                                           "randForce", "randTorque")}
    b["segLength"] = np.zeros(n, F32)
    b["brownTransScale"] = np.zeros(n, F32)
    b["brownRotScale"] = np.zeros(n, F32)
    b["coord64"] = None
    b["n"] = n
    return b


def store_drag(b, i, g):
    """DragTensorSystem.storeDrag (DragTensorSystem.java:61-69)."""
    n = b["n"]
    for k in range(3):
        b["bTransGam"][k * n + i] = F32(g[k])
        b["bRotGam"][k * n + i] = F32(g[3 + k])
        b["bTransDiff"][k * n + i] = F32(KT / g[k])
        b["bRotDiff"][k * n + i] = F32(KT / g[3 + k])


def store_drag_slots(b, idx, g):
    """store_drag for every slot in `idx` (one drag tuple)."""
    n = b["n"]
    idx = np.asarray(idx)
    for k in range(3):
        b["bTransGam"][k * n + idx] = F32(g[k])
        b["bRotGam"][k * n + idx] = F32(g[3 + k])
        b["bTransDiff"][k * n + idx] = F32(KT / g[k])
        b["bRotDiff"][k * n + idx] = F32(KT / g[3 + k])


def set_vec(arr, n, i, x, y, z):
    arr[i] = F32(x)
    arr[n + i] = F32(y)
    arr[2 * n + i] = F32(z)


def derive_host(b):
    """DerivedGeometrySystem.derive over host arrays (float32 arithmetic, as the reference)."""
    n = b["n"]
    u = b["uVec"].reshape(3, n)
    y = b["yVec"].reshape(3, n)
    c = b["coord"].reshape(3, n)
    ux, uy, uz = u
    yx, yy, yz = y
    zx = uy * yz - uz * yy
    zy = uz * yx - ux * yz
    zz = ux * yy - uy * yx
    m2 = zx * zx + zy * zy + zz * zz
    inv = np.where(m2 > 0, F32(1.0) / np.sqrt(np.where(m2 > 0, m2, F32(1))), F32(1)).astype(F32)
    zx = np.where(m2 > 0, zx * inv, zx)
    zy = np.where(m2 > 0, zy * inv, zy)
    zz = np.where(m2 > 0, zz * inv, zz)
    b["zVec"][:] = np.concatenate([zx, zy, zz]).astype(F32)
    b["yVec"][:] = np.concatenate([zy * uz - zz * uy, zz * ux - zx * uz, zx * uy - zy * ux]).astype(F32)
    half = (b["segLength"] * F32(0.5)).astype(F32)
    b["end1"][:] = np.concatenate([c[k] - half * u[k] for k in range(3)]).astype(F32)
    b["end2"][:] = np.concatenate([c[k] + half * u[k] for k in range(3)]).astype(F32)


def filament_store(n):
    """FilamentStore.java:139-199."""
    f = {"body": rigid_body(n)}
    f["monomerCount"] = np.zeros(n, I32)
    for k in ("end1NbrSlot", "end1NbrSide", "end2NbrSlot", "end2NbrSide"):
        f[k] = np.full(n, -1, I32)
    f["filState"] = np.zeros(n, I32)
    f["params"] = np.zeros(2, F32)
    f["counts"] = np.array([n, 0, 0, 1], I32)
    f["chainParams"] = np.zeros(7, F32)
    f["extForce"] = np.zeros(3 * n, F32)
    return f


def drag_run_filament(f, aeta):
    """DragTensorSystem.run(FilamentStore) (DragTensorSystem.java:71-97), viscosity `aeta`."""
    b = f["body"]
    halfmono = ACTIN_MONO_RADIUS
    mono = f["monomerCount"].astype(np.int64)
    at_end = (f["end1NbrSlot"] == -1) | (f["end2NbrSlot"] == -1)
    for m in np.unique(mono):
        length = (int(m) + 1) * ACTIN_MONO_RADIUS
        sel_m = mono == m
        b["segLength"][sel_m] = F32(length)
        for end in (False, True):
            sel = np.flatnonzero(sel_m & (at_end == end))
            if sel.size == 0:
                continue
            min_len = STD_SEG_LENGTH * halfmono if end else 30 * halfmono
            as_if = length if length >= min_len else min_len
            store_drag_slots(b, sel, rod_drag_si(as_if, ACTIN_RADIUS, aeta))


def rescale_viscosity(b, r):
    """DenseContractileHarness.CrosslinkerBundleHarnessAeta (DenseContractileHarness.java:284-290):
    gamma *= r and D /= r, each as (float)((double)value op r)."""
    for k in ("bTransGam", "bRotGam"):
        b[k][:] = (b[k].astype(np.float64) * r).astype(F32)
    for k in ("bTransDiff", "bRotDiff"):
        b[k][:] = (b[k].astype(np.float64) / r).astype(F32)


def set_chain_params(f, dt, frac_move=0.5, frac_r=0.1, frac_move_torq=0.265, spring_active=0.0,
                     spring=1.0e-20):
    """FilamentStore.setChainParams (FilamentStore.java:345-353)."""
    f["chainParams"][:] = np.array([dt, frac_move, frac_r, frac_move_torq, spring_active, spring,
                                    ACTIN_MONO_RADIUS], F32)


# ---------------------------------------------------------------------------- free rods
def free_rods_fdt(n, monomer_ct=64, trans_scale=1.0, rot_scale=0.0, aeta=0.1, dt=1e-4, seed=12345):
    """DiffusionHarness.freshStore (DiffusionHarness.java:742-755): n rods at the origin,
    uVec = +x, yVec = +y; Config T uses (1, 0), Config R uses (0, 1)."""
    f = filament_store(n)
    b = f["body"]
    f["monomerCount"][:] = monomer_ct
    b["uVec"][:n] = 1.0
    b["yVec"][n:2 * n] = 1.0
    b["brownTransScale"][:] = F32(trans_scale)
    b["brownRotScale"][:] = F32(rot_scale)
    drag_run_filament(f, aeta)
    f["params"][:] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    f["counts"][:] = np.array([n, 0, seed, 1], I32)
    return f


def free_rods_box(n=1024, length_um=1.0, radius_um=0.004, box_um=10.0, aeta=1.0e-3, dt=1.0e-5,
                  seed=0x5B0C0, trans_scale=1.0, rot_scale=1.0):
    """Free Brownian rods: centres uniform in a cubic box, orientations uniform on the
    sphere (normalised Gaussian triplet), slender-rod drag for (length, radius) in a
    fluid of viscosity aeta."""
    rng = np.random.default_rng(seed)
    f = filament_store(n)
    b = f["body"]
    c = rng.uniform(0.0, box_um, size=(3, n))
    u = rng.normal(size=(3, n))
    u /= np.linalg.norm(u, axis=0)
    a = np.where(np.abs(u[0]) < 0.9, 0, 1)                 # helper axis not parallel to u
    helper = np.zeros((3, n))
    helper[a, np.arange(n)] = 1.0
    y = helper - (helper * u).sum(0) * u
    y /= np.linalg.norm(y, axis=0)
    b["coord"][:] = c.reshape(-1).astype(F32)
    b["uVec"][:] = u.reshape(-1).astype(F32)
    b["yVec"][:] = y.reshape(-1).astype(F32)
    b["segLength"][:] = F32(length_um)
    g = rod_drag_si(length_um, radius_um, aeta)
    for i in range(n):
        store_drag(b, i, g)
    b["brownTransScale"][:] = F32(trans_scale)
    b["brownRotScale"][:] = F32(rot_scale)
    f["params"][:] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    f["counts"][:] = np.array([n, 0, seed & 0x7FFFFFFF, 1], I32)
    derive_host(b)
    return f


def deflection_chain(n_seg=11, frac_r=0.1, frac_move_torq=0.265, dt=1e-4):
    """DiffusionHarness.measureDeflection set-up (DiffusionHarness.java:287-335): pinned
    11-segment chain, Brownian off, midpoint load F = 48*EI*0.01/span^2."""
    monomer_ct = STD_SEG_LENGTH
    frac = 0.01
    seg_len = (monomer_ct + 1) * ACTIN_MONO_RADIUS
    total = n_seg * seg_len
    span_m = total * 1.0e-6
    force_n = 48.0 * EI * frac / (span_m * span_m)
    mid = n_seg // 2
    f = filament_store(n_seg)
    b = f["body"]
    x0 = -0.5 * total + 0.5 * seg_len
    for k in range(n_seg):
        f["monomerCount"][k] = monomer_ct
        set_vec(b["uVec"], n_seg, k, 1, 0, 0)
        set_vec(b["yVec"], n_seg, k, 0, 1, 0)
        set_vec(b["coord"], n_seg, k, x0 + k * seg_len, 0, 0)
        if k < n_seg - 1:
            f["end2NbrSlot"][k] = k + 1
            f["end2NbrSide"][k] = 0
        if k > 0:
            f["end1NbrSlot"][k] = k - 1
            f["end1NbrSide"][k] = 1
    drag_run_filament(f, 0.1)
    f["params"][:] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    set_chain_params(f, dt)
    f["chainParams"][2] = F32(frac_r)
    f["chainParams"][3] = F32(frac_move_torq)
    f["extForce"][n_seg + mid] = F32(-force_n)
    f["counts"][:] = np.array([n_seg, 0, 1, 1], I32)
    f["pinSeg"] = np.array([0, n_seg - 1], I32)
    f["pinEnd"] = np.array([1, 2], I32)
    f["pinAnchor"] = np.array([-0.5 * total, 0, 0, 0.5 * total, 0, 0], F32)
    f["analyticDefl"] = frac * total
    f["mid"] = mid
    return f


# ---------------------------------------------------------------------------- dense network
@dataclass
class DenseConfig:
    """Composition of a dense contractile network (DenseContractileHarness.java:42-63)."""
    n_fil: int = 2000
    segs_per_fil: int = 10
    monomer_ct: int = 36            # (36+1)*0.0027 um = 0.0999 um rods
    n_mini: int = 200
    dimers_per_end: int = 8         # 16 heads per backbone end
    backbone_len: float = 0.8
    head_zone: float = 0.05
    n_links: int = 4000
    side: float = 20.0
    aspect: float = 1.0              # slab x:y aspect at the same area (side_x = side*sqrt(aspect))
    cell_scale: float = 1.0          # grid cell / the completeness minimum (>= 1; a tuning knob)
    box_z: float = 0.5
    dt: float = 1.0e-5
    aeta: float = 0.1               # Constants.aeta: motors, backbones, and the filament base drag
    fil_aeta: float = 1.0           # DenseContractileHarness.AETA: filament drag rescaled to it
    myo_col_tol: float = 0.030
    align_tol: float = -0.4
    k_off: float = 20.0
    myo_spring: float = 1.0e-9
    j1_fmt: float = 0.4
    brown_trans: float = 1.0
    brown_rot: float = 0.3
    chain_frac_move: float = 0.5
    chain_frac_r: float = 0.1
    chain_frac_move_torq: float = 0.2
    xl_grab: float = 0.05
    xl_rest: float = 0.035
    xl_frac_move: float = 0.4
    xl_off: tuple = (1.0, 0.0, 2.0)  # k_off = c + a*exp(b*strain): 1/s
    xl_torsion_spring: float = 1.0e-19
    xl_unbind: bool = True
    fast_links: bool = False         # seeded KD-tree placement (large scale-sweep networks)
    seed: int = 0x0CDE5
    seed_bb: int = 0x5C2F11
    seed_fil: int = 0xF11A

    @property
    def n_seg(self):
        return self.n_fil * self.segs_per_fil


# The dense contractile network of the benchmark: 2,000 filaments x 10 rods of 0.1 um,
# 200 minifilaments (0.8 um backbone, 16 heads per end), 4,000 crosslinkers, 20x20x0.5 um
# slab with walls, dt = 10 us. Viscosities are the reference dense harness's: filaments in
# the crowded-cytoplasm 1.0 Pa s, myosin bodies at Constants.aeta = 0.1 Pa s (with water,
# the crosslinkers' explicit 1e-19 N m/rad torsion spring turns a 0.1 um rod by about twice
# its misalignment per 10 us step, an unstable explicit update).
C1 = DenseConfig()


def dense_small(scale=0.05, **kw):
    """The same composition scaled down (slab side scaled to keep density)."""
    c = C1
    n_fil = max(2, int(round(c.n_fil * scale)))
    n_mini = max(1, int(round(c.n_mini * scale)))
    n_links = max(1, int(round(c.n_links * scale)))
    side = c.side * math.sqrt(scale)
    return replace(c, n_fil=n_fil, n_mini=n_mini, n_links=n_links, side=side, **kw)


def _place_arm(b, m, rc, d, p, e2, splay, cfg):
    """ContractileAssayHarness.placeArm (ContractileAssayHarness.java:996-1016)."""
    n = b["n"]
    rod, lever, head = 3 * m, 3 * m + 1, 3 * m + 2
    dx, dy, dz = d
    px, py, pz = p
    set_vec(b["coord"], n, rod, *rc)
    set_vec(b["uVec"], n, rod, dx, dy, dz)
    set_vec(b["yVec"], n, rod, px, py, pz)
    lux = COS80 * dx + splay * SIN80 * px
    luy = COS80 * dy + splay * SIN80 * py
    luz = COS80 * dz + splay * SIN80 * pz
    nx, ny, nz = dy * pz - dz * py, dz * px - dx * pz, dx * py - dy * px
    ll, hl = LEVER_LEN, HEAD_LEN
    set_vec(b["coord"], n, lever, e2[0] + 0.5 * ll * lux, e2[1] + 0.5 * ll * luy, e2[2] + 0.5 * ll * luz)
    set_vec(b["uVec"], n, lever, lux, luy, luz)
    set_vec(b["yVec"], n, lever, nx, ny, nz)
    le2 = (e2[0] + ll * lux, e2[1] + ll * luy, e2[2] + ll * luz)
    set_vec(b["coord"], n, head, le2[0] + 0.5 * hl * lux, le2[1] + 0.5 * hl * luy, le2[2] + 0.5 * hl * luz)
    set_vec(b["uVec"], n, head, lux, luy, luz)
    set_vec(b["yVec"], n, head, nx, ny, nz)
    b["brownTransScale"][rod] = F32(cfg.brown_trans)
    b["brownRotScale"][rod] = F32(cfg.brown_rot)
    b["brownTransScale"][lever] = 0
    b["brownRotScale"][lever] = 0
    b["brownTransScale"][head] = F32(cfg.brown_trans)
    b["brownRotScale"][head] = F32(cfg.brown_rot)


def _place_dimer_along(b, mA, mB, e1, d, p, cfg):
    """ContractileAssayHarness.placeDimerAlong (ContractileAssayHarness.java:982-995)."""
    dx, dy, dz = d
    dm = math.sqrt(dx * dx + dy * dy + dz * dz)
    dx, dy, dz = dx / dm, dy / dm, dz / dm
    px, py, pz = p
    pm = math.sqrt(px * px + py * py + pz * pz)
    px, py, pz = px / pm, py / pm, pz / pm
    rl = ROD_LEN
    rc = (e1[0] + 0.5 * rl * dx, e1[1] + 0.5 * rl * dy, e1[2] + 0.5 * rl * dz)
    e2 = (e1[0] + rl * dx, e1[1] + rl * dy, e1[2] + rl * dz)
    _place_arm(b, mA, rc, (dx, dy, dz), (px, py, pz), e2, +1, cfg)
    _place_arm(b, mB, rc, (dx, dy, dz), (px, py, pz), e2, -1, cfg)


def _place_dimers(b, e1, d, p, cfg):
    """_place_dimer_along for every dimer at once (dimer k: motors 2k, 2k+1), the same double
    expressions evaluated elementwise. e1, d, p: (3, nDimers) float64."""
    n = b["n"]
    nd = e1.shape[1]
    dm = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    dx, dy, dz = d[0] / dm, d[1] / dm, d[2] / dm
    pm = np.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
    px, py, pz = p[0] / pm, p[1] / pm, p[2] / pm
    rl = ROD_LEN
    rc = (e1[0] + 0.5 * rl * dx, e1[1] + 0.5 * rl * dy, e1[2] + 0.5 * rl * dz)
    e2 = (e1[0] + rl * dx, e1[1] + rl * dy, e1[2] + rl * dz)
    ll, hl = LEVER_LEN, HEAD_LEN
    nx, ny, nz = dy * pz - dz * py, dz * px - dx * pz, dx * py - dy * px

    def put(arr, slots, x, y, z):
        arr[slots] = np.asarray(x).astype(F32)
        arr[n + slots] = np.asarray(y).astype(F32)
        arr[2 * n + slots] = np.asarray(z).astype(F32)

    for splay, m in ((+1, 2 * np.arange(nd)), (-1, 2 * np.arange(nd) + 1)):
        rod, lever, head = 3 * m, 3 * m + 1, 3 * m + 2
        put(b["coord"], rod, *rc)
        put(b["uVec"], rod, dx, dy, dz)
        put(b["yVec"], rod, px, py, pz)
        lux = COS80 * dx + splay * SIN80 * px
        luy = COS80 * dy + splay * SIN80 * py
        luz = COS80 * dz + splay * SIN80 * pz
        put(b["coord"], lever, e2[0] + 0.5 * ll * lux, e2[1] + 0.5 * ll * luy, e2[2] + 0.5 * ll * luz)
        put(b["uVec"], lever, lux, luy, luz)
        put(b["yVec"], lever, nx, ny, nz)
        le2 = (e2[0] + ll * lux, e2[1] + ll * luy, e2[2] + ll * luz)
        put(b["coord"], head, le2[0] + 0.5 * hl * lux, le2[1] + 0.5 * hl * luy, le2[2] + 0.5 * hl * luz)
        put(b["uVec"], head, lux, luy, luz)
        put(b["yVec"], head, nx, ny, nz)
        b["brownTransScale"][rod] = F32(cfg.brown_trans)
        b["brownRotScale"][rod] = F32(cfg.brown_rot)
        b["brownTransScale"][lever] = 0
        b["brownRotScale"][lever] = 0
        b["brownTransScale"][head] = F32(cfg.brown_trans)
        b["brownRotScale"][head] = F32(cfg.brown_rot)


def _pack_cell(x, y, z):
    return ((x & 0x1FFFFF) << 42) | ((y & 0x1FFFFF) << 21) | (z & 0x1FFFFF)


def dense_contractile(cfg: DenseConfig = C1):
    """DenseContractileHarness.buildScene (DenseContractileHarness.java:112-280) for the
    composition `cfg`. Returns a dict-of-stores scene (host numpy arrays)."""
    rng = JavaRandom(cfg.seed)
    side, box_z, dt = cfg.side, cfg.box_z, cfg.dt
    side_x, side_y = (side, side) if cfg.aspect == 1.0 else (side * math.sqrt(cfg.aspect),
                                                              side / math.sqrt(cfg.aspect))
    n_fil, S = cfg.n_fil, cfg.segs_per_fil
    n_seg = n_fil * S
    n_mini = cfg.n_mini
    n_dimers = n_mini * 2 * cfg.dimers_per_end
    n_mot = 2 * n_dimers
    L = (cfg.monomer_ct + 1) * ACTIN_MONO_RADIUS
    hz = 0.5 * box_z
    margin = 0.5 * (S * L)

    # ---- filaments: free multi-segment chains ----
    f = filament_store(n_seg)
    fb = f["body"]
    # per filament: the reference's four draws, in order; per segment: the same double
    # expressions evaluated elementwise
    fil = np.empty((n_fil, 6))
    for p in range(n_fil):
        cx = (rng.next_double() - 0.5) * (side_x - 2 * margin)
        cy = (rng.next_double() - 0.5) * (side_y - 2 * margin)
        cz = (rng.next_double() - 0.5) * (box_z - 0.1)
        th = rng.next_double() * math.pi * 2
        fil[p] = (cx, cy, cz, math.cos(th), math.sin(th), 0.0)
    off = (np.arange(S) - 0.5 * (S - 1)) * L
    cx, cy, cz, ux, uy, uz = (np.repeat(fil[:, k], S) for k in range(6))
    offs = np.tile(off, n_fil)
    f["monomerCount"][:] = cfg.monomer_ct
    fb["uVec"][:] = np.concatenate([ux, uy, uz]).astype(F32)
    fb["yVec"][:] = np.concatenate([-uy, ux, np.zeros(n_seg)]).astype(F32)
    fb["coord"][:] = np.concatenate([cx + offs * ux, cy + offs * uy, cz + offs * uz]).astype(F32)
    fb["brownTransScale"][:] = F32(BTRANS_COEFF)
    sidx = np.tile(np.arange(S), n_fil)
    ends = (sidx == 0) | (sidx == S - 1)
    fb["brownRotScale"][:] = np.where(ends, F32(BROT_COEFF), F32(0.0)).astype(F32)
    g = np.arange(n_seg)
    inner2 = sidx < S - 1
    f["end2NbrSlot"][inner2] = g[inner2] + 1
    f["end2NbrSide"][inner2] = 0
    inner1 = sidx > 0
    f["end1NbrSlot"][inner1] = g[inner1] - 1
    f["end1NbrSide"][inner1] = 1
    drag_run_filament(f, cfg.aeta)
    if cfg.fil_aeta != cfg.aeta:
        rescale_viscosity(fb, cfg.fil_aeta / cfg.aeta)
    f["params"][:] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    f["counts"][:] = np.array([n_seg, 0, cfg.seed_fil, 1], I32)
    f["chainParams"][:] = np.array([dt, cfg.chain_frac_move, cfg.chain_frac_r, cfg.chain_frac_move_torq,
                                    0.0, 1.0e-20, ACTIN_MONO_RADIUS], F32)
    derive_host(fb)

    # ---- minifilaments: backbones each owning 2*dimers_per_end splayed dimers ----
    mot = {"body": rigid_body(3 * n_mot), "nMotors": n_mot}
    mb = mot["body"]
    dim = {"nDimers": n_dimers, "motorA": np.zeros(n_dimers, I32), "motorB": np.zeros(n_dimers, I32),
           "parallel": np.ones(n_dimers, I32)}
    mini = {"backbone": rigid_body(n_mini), "nBackbones": n_mini, "nDimers": n_dimers,
            "headBackboneSlot": np.zeros(n_dimers, I32), "motorA": np.zeros(n_dimers, I32),
            "attachAxial": np.zeros(n_dimers, F32), "miniData": np.zeros(MINI_STRIDE * n_dimers, F32),
            "bbInvDragY": np.zeros(2 * n_mini, F32), "bbDimerCount": np.zeros(n_mini, I32),
            "bbDimerOffsets": np.zeros(n_mini + 1, I32), "bbDimerList": np.zeros(n_dimers, I32)}
    bbb = mini["backbone"]
    reach = np.zeros(n_mot, F32)
    d = 0
    dimer_rows = []
    for mfi in range(n_mini):
        bx = (rng.next_double() - 0.5) * (side_x - 2 * margin)
        by = (rng.next_double() - 0.5) * (side_y - 2 * margin)
        bz = (rng.next_double() - 0.5) * (box_z - 0.1)
        th = rng.next_double() * math.pi * 2
        ux, uy, uz = math.cos(th), math.sin(th), 0.0
        yx, yy, yz = -uy, ux, 0.0
        set_vec(bbb["coord"], n_mini, mfi, bx, by, bz)
        set_vec(bbb["uVec"], n_mini, mfi, ux, uy, uz)
        set_vec(bbb["yVec"], n_mini, mfi, yx, yy, yz)
        bbb["brownTransScale"][mfi] = F32(cfg.brown_trans)
        bbb["brownRotScale"][mfi] = F32(cfg.brown_rot)
        for e in range(2):
            sgn = -1.0 if e == 0 else 1.0
            for j in range(cfg.dimers_per_end):
                mag = cfg.backbone_len / 2.0 - (j + 0.5) / cfg.dimers_per_end * cfg.head_zone
                ax = sgn * mag
                phi = (j + 0.5) / cfg.dimers_per_end * math.pi
                dimer_rows.append((bx + ax * ux, by + ax * uy, bz + ax * uz, sgn * ux, sgn * uy, sgn * uz,
                                   math.cos(phi) * yx + math.sin(phi) * (uy * yz - uz * yy),
                                   math.cos(phi) * yy + math.sin(phi) * (uz * yx - ux * yz),
                                   math.cos(phi) * yz + math.sin(phi) * (ux * yy - uy * yx), ax, mfi))
                d += 1
    if n_dimers:
        rows = np.array(dimer_rows)
        _place_dimers(mb, rows[:, 0:3].T, rows[:, 3:6].T, rows[:, 6:9].T, cfg)
        dd = np.arange(n_dimers)
        dim["motorA"][:], dim["motorB"][:], dim["parallel"][:] = 2 * dd, 2 * dd + 1, 1
        mini["headBackboneSlot"][:] = rows[:, 10].astype(I32)
        mini["motorA"][:] = 2 * dd
        mini["attachAxial"][:] = rows[:, 9].astype(F32)
        reach[:] = F32(cfg.myo_col_tol)
    # DragTensorSystem.run(MotorStore) (DragTensorSystem.java:105-122)
    gr = rod_drag_si(ROD_LEN, ROD_R, cfg.aeta)
    gl = rod_drag_si(LEVER_LEN, LEVER_R, cfg.aeta)
    gh = sphere_drag_si(HEAD_R, cfg.aeta)
    mb["segLength"][0::3] = F32(ROD_LEN)
    mb["segLength"][1::3] = F32(LEVER_LEN)
    mb["segLength"][2::3] = F32(HEAD_LEN)
    store_drag_slots(mb, np.arange(n_mot) * 3, gr)
    store_drag_slots(mb, np.arange(n_mot) * 3 + 1, gl)
    store_drag_slots(mb, np.arange(n_mot) * 3 + 2, gh)
    # MiniFilamentStore.initBackboneDrag (MiniFilamentStore.java:121-134)
    gbb = rod_drag_si(cfg.backbone_len, BACKBONE_R, cfg.aeta)
    bbb["segLength"][:] = F32(cfg.backbone_len)
    store_drag_slots(bbb, np.arange(n_mini), gbb)
    mini["bbInvDragY"][:n_mini] = F32(1.0 / gbb[1])
    mini["bbInvDragY"][n_mini:] = F32(1.0 / gbb[4])

    # MotorStore set-up (MotorStore.java:190-263), DenseContractileHarness.java:210-215
    mot.update({
        "head": np.zeros(3 * n_mot, F32), "uVec": np.zeros(3 * n_mot, F32), "rodUVec": np.zeros(3 * n_mot, F32),
        "reach": reach, "boundSeg": np.full(n_mot, -1, I32), "bindArc": np.zeros(n_mot, F32),
        "stats": np.zeros(2 * n_mot, I32), "capStats": np.zeros(n_mot, I32), "cooldown": np.zeros(n_mot, I32),
        "nucleotideState": np.zeros(n_mot, I32), "forceDotPlace": np.zeros(n_mot, I32),
        "forceDotFil": np.zeros(n_mot, F32), "forceMag": np.zeros(n_mot, F32),
        "forceDotHist": np.zeros(10 * n_mot, F32),
        "bodyParams": np.array([dt, math.sqrt(2.0 * KT / dt)], F32),
        "jointParams": np.array([dt, 0.4, 0.4, 0.4, 0.0, 0.4, 0.4, 0.0, 96.0, 0.4, 6.0], F32),
        "kinParams": np.array([cfg.k_off, 0.92, 0.08, 2.5e-9, 0.4e-9, KT, dt, cfg.myo_col_tol, cfg.align_tol,
                               0.0, math.ceil(MYO_REBIND_TIME / dt), 12.0e-12, 1.0, 1.0], F32),
        "nucParams": np.array([dt, 2.0e4, 100.0, 100.0, 1.0e4, 0.0, 1.0e3, 1.0e3], F32),
        "counts": np.array([n_mot, 0, cfg.seed, n_seg], I32),
        "publishParams": np.array([n_seg], I32),
    })
    dim["dimerParams"] = np.array([dt, DIMER_ROD_FRAC_MOVE, DIMER_LEVER_FMT, DIMER_LEVER_DEG, ROD_LEN], F32)
    mini["miniParams"] = np.array([dt, MINIFIL_FRAC_MOVE, MINIFIL_ALIGN], F32)
    mini["bbBodyParams"] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    mini["bbCounts"] = np.array([n_mini, 0, cfg.seed_bb, n_mini], I32)

    # ---- grid + body view (filaments + heads) ----
    cap = n_seg + n_mot
    seg_bound_r = 0.5 * L + ACTIN_RADIUS
    cutoff = cfg.myo_col_tol + 0.5 * ROD_LEN
    cell = 2.0 * seg_bound_r + cutoff
    if cfg.cell_scale != 1.0:
        cell *= max(1.0, cfg.cell_scale)
    gx = 0.5 * side_x + 1.0
    gy = 0.5 * side_y + 1.0
    gz = hz + 0.3
    nX = 1 + int(math.ceil(2 * gx / cell))
    nY = 1 + int(math.ceil(2 * gy / cell))
    nZ = 1 + int(math.ceil(2 * gz / cell))
    total_cells = nX * nY * nZ
    grid = {
        "cap": cap, "totalCells": total_cells,
        "center": np.zeros(3 * cap, F32), "boundingRadius": np.zeros(cap, F32),
        "ownerStore": np.full(cap, -1, I32), "ownerSlot": np.full(cap, -1, I32),
        "gridParams": np.array([-gx, -gy, -gz, cell, 1.0 / cell, cutoff], F32),
        "viewParams": np.array([ACTIN_RADIUS], F32),
        "gridDims": np.array([nX, nY, nZ, total_cells], I32),
        "gridCounts": np.array([0, cap, 0, 0], I32),
        "bodyCell": np.full(cap, -1, I32), "cellCount": np.zeros(total_cells, I32),
        "chunkSum": np.zeros((total_cells + GRID_SCAN_CHUNK - 1) // GRID_SCAN_CHUNK + 1, I32),
        "gridCellOffsets": np.zeros(total_cells + 1, I32), "gridCellContents": np.full(cap, -1, I32),
        "reachSeg": np.full(n_mot * MAX_CAND, -1, I32), "reachCount": np.zeros(n_mot, I32),
    }

    # ---- crosslinkers pre-placed between nearby segments of distinct filaments ----
    xl = _build_crosslinkers_fast(f, n_seg, S, cfg) if cfg.fast_links else _build_crosslinkers(f, n_seg, S, cfg, rng)

    check_int = max(1, int(round(1.0e-4 / dt)))
    scene = {
        "cfg": cfg, "fil": f, "mot": mot, "dim": dim, "mini": mini, "xl": xl, "grid": grid,
        "bondData": np.zeros(n_mot * XB_STRIDE, F32),
        "xbParams": np.array([cfg.myo_spring, 90.0, cfg.j1_fmt, dt, HEAD_LEN, 0.0], F32),
        "boxParams": np.array([1.0e-4, side_x, side_y, box_z, ACTIN_RADIUS, 0.5, check_int, dt], F32),
        "segMotorCount": np.zeros(n_seg, I32), "segMotorOffsets": np.zeros(n_seg + 1, I32),
        "segMotorMyo": np.zeros(n_mot, I32),
        "seed": cfg.seed, "seedBb": cfg.seed_bb, "xlinkOn": 1, "xlUnbind": 1 if cfg.xl_unbind else 0,
    }
    return scene


def _build_crosslinkers(f, n_seg, segs_per_fil, cfg, rng):
    """DenseContractileHarness.buildCrosslinkers (DenseContractileHarness.java:296-341)."""
    n_links = cfg.n_links
    xl = {"nLinks": n_links,
          "linkFilA": np.full(n_links, -1, I32), "linkFilB": np.full(n_links, -1, I32),
          "linkState": np.full(n_links, -1, I32), "linkOrientSame": np.zeros(n_links, I32),
          "activeLinkCount": np.zeros(n_seg, I32),
          "loc1": np.zeros(n_links, F32), "loc2": np.zeros(n_links, F32),
          "xlinkData": np.zeros(n_links * XL_STRIDE, F32),
          "strainHist": np.zeros(n_links * STRAIN_WIN, F32), "torqueMagHist": np.zeros(n_links * TORQUE_WIN, F32),
          "strainPlace": np.zeros(n_links, I32), "torqueMagPlace": np.zeros(n_links, I32),
          "counts": np.array([n_links, 0, 0, n_seg], I32)}
    for k in ("segCountA", "segCountB"):
        xl[k] = np.zeros(n_seg, I32)
    for k in ("segOffsetsA", "segOffsetsB"):
        xl[k] = np.zeros(n_seg + 1, I32)
    for k in ("segIdxA", "segIdxB"):
        xl[k] = np.zeros(n_links, I32)
    fb = f["body"]
    c = fb["coord"]
    grab = cfg.xl_grab
    cell = grab
    buckets = {}
    cx_all = np.floor(c[:n_seg].astype(np.float64) / cell).astype(np.int64)
    cy_all = np.floor(c[n_seg:2 * n_seg].astype(np.float64) / cell).astype(np.int64)
    cz_all = np.floor(c[2 * n_seg:].astype(np.float64) / cell).astype(np.int64)
    for s in range(n_seg):
        buckets.setdefault(_pack_cell(int(cx_all[s]), int(cy_all[s]), int(cz_all[s])), []).append(s)
    placed = attempts = 0
    while placed < n_links and attempts < n_links * 200:
        attempts += 1
        s = rng.next_int(n_seg)
        fil_s = s // segs_per_fil
        sx, sy, sz = float(c[s]), float(c[n_seg + s]), float(c[2 * n_seg + s])
        best, best_d = -1, grab * grab
        cx, cy, cz = math.floor(sx / cell), math.floor(sy / cell), math.floor(sz / cell)
        dx = -1
        while dx <= 1 and best < 0:
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    bucket = buckets.get(_pack_cell(cx + dx, cy + dy, cz + dz))
                    if bucket is None:
                        continue
                    for t in bucket:
                        if t // segs_per_fil == fil_s:
                            continue
                        ddx = float(c[t]) - sx
                        ddy = float(c[n_seg + t]) - sy
                        ddz = float(c[2 * n_seg + t]) - sz
                        dd = ddx * ddx + ddy * ddy + ddz * ddz
                        if dd < best_d:
                            best_d, best = dd, t
            dx += 1
        if best < 0:
            continue
        xl["linkFilA"][placed] = s
        xl["linkFilB"][placed] = best
        xl["loc1"][placed] = F32(0.5 * float(fb["segLength"][s]))
        xl["loc2"][placed] = F32(0.5 * float(fb["segLength"][best]))
        xl["linkState"][placed] = 0
        xl["linkOrientSame"][placed] = 1
        placed += 1
    xl["placed"] = placed
    xl["xlParams"] = np.array([cfg.xl_rest, cfg.xl_frac_move, cfg.dt], F32)
    xl["offParams"] = np.array([cfg.xl_off[0], cfg.xl_off[1], cfg.xl_off[2], cfg.dt, cfg.xl_rest], F32)
    xl["torsionParams"] = np.array([cfg.xl_torsion_spring, 1.0], F32)
    xl["counts"][2] = cfg.seed
    return xl


def _build_crosslinkers_fast(f, n_seg, segs_per_fil, cfg):
    """The composition of buildCrosslinkers for large networks: each link joins a random
    segment to the nearest segment of another filament within the grab distance, found with
    a KD-tree; draws from a seeded numpy generator (not the harness's java.util.Random
    sequence), so the network differs from the exact builder's but has its statistics."""
    from scipy.spatial import cKDTree
    n_links = cfg.n_links
    proto = _build_crosslinkers(f, n_seg, segs_per_fil, replace(cfg, n_links=0), None)
    xl = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in proto.items()}
    for k, shape, fill, dt in (("linkFilA", n_links, -1, I32), ("linkFilB", n_links, -1, I32),
                               ("linkState", n_links, -1, I32), ("linkOrientSame", n_links, 0, I32),
                               ("loc1", n_links, 0, F32), ("loc2", n_links, 0, F32),
                               ("xlinkData", n_links * XL_STRIDE, 0, F32), ("strainHist", n_links * STRAIN_WIN, 0, F32),
                               ("torqueMagHist", n_links * TORQUE_WIN, 0, F32), ("strainPlace", n_links, 0, I32),
                               ("torqueMagPlace", n_links, 0, I32), ("segIdxA", n_links, 0, I32),
                               ("segIdxB", n_links, 0, I32)):
        xl[k] = np.full(shape, fill, dt)
    xl["nLinks"] = n_links
    xl["counts"][0] = n_links
    fb = f["body"]
    pts = np.stack([fb["coord"][:n_seg], fb["coord"][n_seg:2 * n_seg], fb["coord"][2 * n_seg:]], 1).astype(np.float64)
    fil = np.arange(n_seg) // segs_per_fil
    tree = cKDTree(pts)
    rng = np.random.default_rng(cfg.seed)
    placed = 0
    while placed < n_links:
        draws = rng.integers(0, n_seg, size=2 * (n_links - placed) + 64)
        dist, idx = tree.query(pts[draws], k=24, distance_upper_bound=cfg.xl_grab)
        ok = (idx < n_seg)
        ok &= fil[np.minimum(idx, n_seg - 1)] != fil[draws][:, None]
        has = ok.any(1)
        first = np.argmax(ok, 1)
        for r in np.flatnonzero(has):
            if placed == n_links:
                break
            a, b = int(draws[r]), int(idx[r, first[r]])
            xl["linkFilA"][placed], xl["linkFilB"][placed] = a, b
            xl["loc1"][placed] = F32(0.5 * float(fb["segLength"][a]))
            xl["loc2"][placed] = F32(0.5 * float(fb["segLength"][b]))
            xl["linkState"][placed] = 0
            xl["linkOrientSame"][placed] = 1
            placed += 1
    xl["placed"] = placed
    return xl


def dense_scaled(n_rods, **kw):
    """The benchmark network's composition at `n_rods` actin rods and the same density
    (the scale sweep: slab side scaled by sqrt(n_rods / 20,000)), crosslinkers placed by
    the KD-tree builder."""
    c = C1
    scale = n_rods / c.n_seg
    return replace(c, n_fil=int(n_rods) // c.segs_per_fil, n_mini=max(1, int(round(c.n_mini * scale))),
                   n_links=max(1, int(round(c.n_links * scale))), side=c.side * math.sqrt(scale), fast_links=True,
                   **kw)


# ---------------------------------------------------------------- crosslinker formation scene
XL_BUNDLE_REST_LEN = 0.0125                  # CrosslinkerBundleHarness.java:46 (FilLink.restLength)
XL_GRAB_DIST = 2.0 * 0.0054                  # crossLinkGrabDist = 2 actinMonoDiam (:51)
XL_MIN_SEP = 5.0 * 0.0054                    # minSepBetweenXLinks (:52)
XL_MIN_FILLINK_SEP = 2.0 * 0.0054            # loc jitter half-range (:53)
XL_MAX_LINKS_ON_SEG = 10                     # (:54)


def xlink_form_params(max_angle, p_form, grab=XL_GRAB_DIST, min_sep=XL_MIN_SEP, max_links=XL_MAX_LINKS_ON_SEG,
                      jitter=XL_MIN_FILLINK_SEP):
    """CrosslinkerStore.setFormParams (CrosslinkerStore.java:190-199)."""
    return np.array([max_angle, grab * grab, min_sep, max_links, p_form, jitter, grab, 0.0], F32)


def xlink_bundle(n_fil=200, box=(0.7, 0.7, 0.3), dt=1.0e-4, seed=7, pos_sigma=0.2, max_angle=0.6, p_form=0.5,
                 aeta=1.0, mode=0):
    """A dense bundle of single-segment filaments for crosslinker formation, composed like
    CrosslinkerBundleHarness.buildBundle (CrosslinkerBundleHarness.java:260-311): lengths
    uniform in [0.1, 0.3] um, directions uniform on the sphere, centres Gaussian (sigma
    0.2 um) clamped to the box, filID = index, an empty link pool of max(64, 4 n) slots and
    all-pairs request capacity. Seeded numpy draws stand in for java.util.Random."""
    rng = np.random.default_rng(seed)
    n = n_fil
    f = filament_store(n)
    b = f["body"]
    lens = 0.1 + rng.random(n) * 0.2
    f["monomerCount"][:] = np.maximum(1, np.rint(lens / ACTIN_MONO_RADIUS).astype(np.int64) - 1).astype(I32)
    z = 2.0 * rng.random(n) - 1.0
    phi = 2.0 * math.pi * rng.random(n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    u = np.stack([r * np.cos(phi), r * np.sin(phi), z])
    y = np.stack([-u[1], u[0], np.zeros(n)])
    yn = np.linalg.norm(y, axis=0)
    small = yn < 1e-9
    y[:, small] = np.stack([np.zeros(small.sum()), -u[2, small], u[1, small]])
    y /= np.linalg.norm(y, axis=0)
    c = np.stack([np.clip(rng.normal(size=n) * pos_sigma, -0.5 * bx, 0.5 * bx) for bx in box])
    b["coord"][:] = c.reshape(-1).astype(F32)
    b["uVec"][:] = u.reshape(-1).astype(F32)
    b["yVec"][:] = y.reshape(-1).astype(F32)
    b["brownTransScale"][:] = F32(1.0)
    b["brownRotScale"][:] = F32(0.5)
    drag_run_filament(f, 0.1)
    rescale_viscosity(b, aeta / 0.1)
    f["params"][:] = np.array([dt, math.sqrt(2.0 * KT / dt)], F32)
    f["counts"][:] = np.array([n, 0, seed, 1], I32)
    derive_host(b)
    C = max(64, 4 * n)
    req_cap = max(1, n * (n - 1) // 2)
    xl = {"nLinks": C,
          "linkFilA": np.full(C, -1, I32), "linkFilB": np.full(C, -1, I32),
          "linkState": np.full(C, -1, I32), "linkOrientSame": np.zeros(C, I32),
          "activeLinkCount": np.zeros(n, I32),
          "loc1": np.zeros(C, F32), "loc2": np.zeros(C, F32),
          "xlinkData": np.zeros(C * XL_STRIDE, F32),
          "strainHist": np.zeros(C * STRAIN_WIN, F32), "torqueMagHist": np.zeros(C * TORQUE_WIN, F32),
          "strainPlace": np.zeros(C, I32), "torqueMagPlace": np.zeros(C, I32),
          "counts": np.array([C, 0, seed, n], I32),
          "reqFilA": np.full(req_cap, -1, I32), "reqFilB": np.full(req_cap, -1, I32),
          "reqLoc1": np.zeros(req_cap, F32), "reqLoc2": np.zeros(req_cap, F32),
          "reqOrient": np.zeros(req_cap, I32), "gatePass": np.zeros(req_cap, I32),
          "acceptFlag": np.zeros(req_cap, I32), "rankOffsets": np.zeros(req_cap + 1, I32),
          "minCand": np.zeros(n, I32),
          "freeCount": np.zeros(C, I32), "freeOffsets": np.zeros(C + 1, I32), "freeList": np.zeros(C, I32),
          "formParams": xlink_form_params(max_angle, p_form),
          "formCounts": np.array([0, 0, seed, mode], I32)}
    seg_len = b["segLength"].astype(np.float64)
    max_c = float(np.abs(b["coord"]).max())
    cell = 2.0 * (0.5 * float(seg_len.max()) + ACTIN_RADIUS) + XL_GRAB_DIST
    g = max(2.0, max_c * 4.0 + cell + 0.5)
    grid = {"half": g, "cell": cell, "grab": XL_GRAB_DIST, "radius": ACTIN_RADIUS}
    return {"fil": f, "xl": xl, "filID": np.arange(n, dtype=I32), "grid": grid, "reqCap": req_cap, "C": C}


# ---------------------------------------------------------------- turnover scene
def turnover_chains(n_chains=200, cap=2048, seg_range=(1, 8), seed=5, cfg=None, tip_mono=(30, 64),
                    body_mono=(2, 40), cofilin_high=0.0):
    """Formin-pinned actin chains for the turnover path, in the harness's chain convention
    (FullSystemDemoHarness.placeRandomChain, :580-606): segment 0 of chain k is the barbed
    tip (seedNode = k, end2 free), segment i's end1 glues to segment i+1's end2, the last
    segment is the pointed tip (end1 free). Chains take random slots of a store of capacity
    `cap`; the other slots are FREE (state -1, zero Brownian scale, monomerCount 0).

    Random, seeded: chain lengths in seg_range, tip monomer counts in tip_mono (64 = at the
    split threshold), other segments in body_mono (below actinSeed = 3 they die at their
    first cadence as a pointed tip), nucleotide compositions summing to 1, cofilin fractions
    up to f_ADP (raised by `cofilin_high` on a tenth of the segments, so that dissolves fire)."""
    from .turnover import TurnoverConfig, turnover_arrays
    cfg = cfg or TurnoverConfig()
    rng = np.random.default_rng(seed)
    lens = rng.integers(seg_range[0], seg_range[1] + 1, n_chains)
    n_used = int(lens.sum())
    if n_used > cap:
        raise ValueError(f"{n_used} segments do not fit capacity {cap}")
    f = filament_store(cap)
    b = f["body"]
    slots = rng.permutation(cap)[:n_used].astype(I32)
    seedNode = np.full(cap, -1, I32)
    mono = np.zeros(cap, I32)
    f["filState"][:] = -1
    pos = 0
    for k in range(n_chains):
        sl = slots[pos:pos + lens[k]]
        pos += lens[k]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        p = np.cross(d, [0.0, 0.0, 1.0] if abs(d[2]) < 0.9 else [1.0, 0.0, 0.0])
        p /= np.linalg.norm(p)
        e = rng.uniform(-2.0, 2.0, 3)
        for i, s in enumerate(sl):
            m = int(rng.integers(tip_mono[0], tip_mono[1] + 1)) if i == 0 else int(
                rng.integers(body_mono[0], body_mono[1] + 1))
            mono[s] = m
            L = (m + 1) * ACTIN_MONO_RADIUS
            c = e + 0.5 * L * d
            set_vec(b["coord"], cap, s, *c)
            set_vec(b["uVec"], cap, s, *d)
            set_vec(b["yVec"], cap, s, *p)
            e = e + L * d
            f["filState"][s] = 0
            b["brownTransScale"][s] = F32(BTRANS_COEFF)
            b["brownRotScale"][s] = F32(BROT_COEFF if i in (0, lens[k] - 1) else 0.0)
            if i == 0:
                seedNode[s] = k
            if i > 0:
                f["end2NbrSlot"][s], f["end2NbrSide"][s] = sl[i - 1], 0
            if i < lens[k] - 1:
                f["end1NbrSlot"][s], f["end1NbrSide"][s] = sl[i + 1], 1
    f["monomerCount"][:] = mono
    free = f["filState"] < 0
    drag_run_filament(f, 0.1)
    b["segLength"][free] = F32(0)
    derive_host(b)
    a = rng.uniform(0.0, 1.0, cap).astype(F32)
    bb = (rng.uniform(0.0, 1.0, cap).astype(F32) * (F32(1) - a)).astype(F32)
    nuc = np.concatenate([a, bb, (F32(1) - a - bb).astype(F32)]).astype(F32)
    adp = nuc[2 * cap:]
    cof = (rng.uniform(0.0, 1.0, cap).astype(F32) * adp).astype(F32)
    if cofilin_high > 0:
        hi = rng.random(cap) < 0.1
        cof[hi] = np.minimum(F32(1), cof[hi] + F32(cofilin_high)).astype(F32)
    t = turnover_arrays(cap, cfg, seedNode=seedNode, nucFrac=nuc, cofFrac=cof)
    return {"fil": f, "t": t, "cfg": cfg, "C": cap, "n_chains": n_chains}


def dense_turnover(cfg=None, growth_rate=10.0, sever_rate=0.01, cof_ratio=0.5, birth_cap=None, seed_mon=None,
                   seed=0x7A11, turnover_seed=None):
    """The dense network with actin turnover on (the scale sweep's turnover workload):

    * growth at every filament's barbed terminal (the end2-free segment, tagged as a
      growing tip in seedNode) at `growth_rate` subunits/s: GrowthSystem's probability
      k_on [actin] biochemDeltaT with the initial [actin] = growth_rate / k_on;
    * severing at `sever_rate` per rod per second through the reference's cofilin rule: an
      aged network (f_ADP = 1) whose cofilin fractions are spread so that -ln(1 - f_cof) is
      uniform on [0, -ln(1 - ratio)), with p_cof chosen so that a rod takes 1/sever_rate
      seconds from f_cof = 0 to the ratio: each rod dissolves once per 1/sever_rate s;
    * pointed-end depolymerisation at the ADP off-rate (depolyProxy);
    * constant-actin births: when depolymerisation and dissolves have returned more
      monomers than growth took, newborn one-rod filaments of `seed_mon` monomers (default:
      the network's rod size) appear at uniform positions in the slab, in dead slots.

    Turnover semantics of a free-filament network are not the reference's (its growth is
    node-bonded and it has no random birth), so this workload is specified here."""
    from .turnover import (BIOCHEM_DT, K_ATP_ON2_WITH_FORMIN, TurnoverConfig, birth_arrays, turnover_arrays)
    cfg = cfg or C1
    sc = dense_contractile(cfg)
    f = sc["fil"]
    n = f["body"]["n"]
    kw = {} if turnover_seed is None else {"seed": int(turnover_seed)}
    tcfg = TurnoverConfig(dt=cfg.dt, cof_ratio=cof_ratio, pool0_um=growth_rate / K_ATP_ON2_WITH_FORMIN, **kw,
                          box_vol_um3=float(sc["boxParams"][1]) * float(sc["boxParams"][2]) * cfg.box_z,
                          aeta=cfg.fil_aeta, born_trans=cfg.brown_trans,
                          born_rot=BROT_COEFF)
    seedNode = np.full(n, -1, I32)
    tips = np.flatnonzero(f["end2NbrSlot"] < 0)
    seedNode[tips] = np.arange(tips.size, dtype=I32)
    nuc = np.zeros(3 * n, F32)
    nuc[2 * n:] = 1.0
    rng = np.random.default_rng(seed)
    x_star = -math.log(1.0 - cof_ratio)
    x0 = rng.uniform(0.0, x_star, n)
    cof = (1.0 - np.exp(-x0)).astype(F32)
    t = turnover_arrays(n, tcfg, seedNode=seedNode, nucFrac=nuc, cofFrac=cof)
    if sever_rate > 0:
        cadences = (1.0 / sever_rate) / BIOCHEM_DT
        t["cofilinParams"][0] = F32(-math.expm1(-x_star / cadences))
    else:                                   # no severing: cofilin stays where it is
        t["cofilinParams"][0] = F32(0.0)
    seed_mon = cfg.monomer_ct if seed_mon is None else seed_mon
    birth_cap = birth_cap or max(64, n // 50)
    bp = sc["boxParams"]
    birth_arrays(t, birth_cap, (0.5 * float(bp[1]), 0.5 * float(bp[2]), 0.5 * cfg.box_z), seed_mon)
    sc["turnover"] = t
    sc["tcfg"] = tcfg
    return sc
