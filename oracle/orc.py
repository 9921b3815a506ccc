"""ctypes wrapper of the oracle (liborc.so).

TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference's DDGI
probe-update path that the CUDA library is checked against, and the FP32 CPU
baseline bench.py times. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs may import it. Parity against the reference itself is
unpinned (see orc_core.hpp).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"
_lib = None


def build() -> Path:
    srcs = list(HERE.glob("*.hpp")) + list(HERE.glob("*.cpp"))
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


class OrcScene(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p), ("nodeCount", C.c_uint32), ("triIndex", C.c_void_p), ("triCount", C.c_uint32),
        ("vertexData", C.c_void_p), ("vertexCount", C.c_uint32), ("triMaterial", C.c_void_p),
        ("materials", C.c_void_p), ("materialsLen", C.c_uint32),
        ("instBase", C.c_uint32), ("instCount", C.c_uint32), ("tlasBase", C.c_uint32), ("tlasNodeCount", C.c_uint32),
    ]


class OrcLights(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dataLen", C.c_uint32), ("lightCount", C.c_uint32), ("clustered", C.c_int32),
                ("emitterBase", C.c_uint32), ("emitterCount", C.c_uint32)]


class OrcGrid(C.Structure):
    _fields_ = [("gridMin", C.c_double * 3), ("gridSize", C.c_double * 3), ("res", C.c_uint32 * 3),
                ("rays", C.c_uint32), ("maxDist", C.c_double), ("cellMin", C.c_double)]


class OrcSolveIO(C.Structure):
    _fields_ = [("rayOut", C.c_void_p), ("hitTri", C.c_void_p), ("hitInst", C.c_void_p), ("secondT", C.c_void_p),
                ("tested", C.c_void_p), ("blocked", C.c_void_p), ("replayTri", C.c_void_p),
                ("replayInst", C.c_void_p), ("replayBlocked", C.c_void_p), ("rayIn", C.c_void_p),
                ("preRound", C.c_void_p), ("counters", C.c_void_p), ("hitFacing", C.c_void_p),
                ("emitterVis", C.c_void_p), ("emitterVisReplay", C.c_void_p), ("emitterSampleOut", C.c_void_p),
                ("reflectTier", C.c_uint32), ("glossyPhase", C.c_uint32), ("roughSpec", C.c_void_p),
                ("roughAtlas", C.c_void_p), ("glossyNum", C.c_void_p), ("glossyDen", C.c_void_p),
                ("glossyAtlas", C.c_void_p)]


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        P, U = C.c_void_p, C.c_uint32
        sig = {
            "orc_version": (C.c_int, []),
            "orc_closest": (None, [P, P, P, U, C.c_int32, C.c_int32, P, P, P, P, C.c_int32]),
            "orc_any": (None, [P, P, P, P, U, P, C.c_int32]),
            "orc_solve_f64": (C.c_int, [P, P, P, P, P, U, U, P, P, P, P, P, C.c_int32]),
            "orc_solve_f32": (C.c_int, [P, P, P, P, P, U, U, P, P, P, P, P, C.c_int32]),
            "orc_params_size": (U, []),
            "orc_light_grid": (None, [P, P, U, P, C.c_int32]),
            "orc_oct_encode": (None, [P, P]),
            "orc_oct_decode": (None, [P, P]),
            "orc_to_half": (C.c_uint16, [C.c_double]),
            "orc_from_half": (C.c_double, [C.c_uint16]),
            "orc_ray_dir": (None, [U, U, C.c_double, P]),
            "orc_probe_world_pos": (None, [P, U, P]),
            "orc_hysteresis_exponent": (C.c_double, [C.c_double, C.c_int32]),
            "orc_grid_resolution": (None, [P, C.c_int32, P]),
            "orc_gutter_source_lane": (C.c_int32, [C.c_int32]),
            "orc_sample_atlas": (None, [P, P, P, P, P]),
            "orc_refit_blas": (C.c_int32, [P, C.c_uint64, P, C.c_uint64, P, C.c_uint64, C.c_int64, C.c_int64]),
            "orc_refit_tlas_range": (C.c_int32, [P, C.c_uint64, P, C.c_uint64, C.c_int64, C.c_int64]),
            "orc_refit_tlas_dirty": (C.c_int32, [P, C.c_uint64, P, C.c_uint64, C.c_int64, P, C.c_uint64, P, P]),
            "orc_build_tlas": (U, [P, U, P, P, P]),
            "orc_compute_instances": (None, [P, P, P, U, P, P, P]),
            "orc_probe_rays": (None, [P, C.c_double, U, U, P, P]),
            "orc_explain_hits": (None, [P, P, P, U, P, P, P, P, P, P, P, C.c_int32]),
            "orc_gather": (None, [P, P, P, P, P, P, P, P, P, P, U, P, P, C.c_int32]),
            "orc_gather_params_size": (U, []),
            "orc_pair_t": (None, [P, P, P, U, P, P, P, C.c_int32]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def threads() -> int:
    return max(1, os.cpu_count() or 1)


# ------------------------------------------------------------ scene tail
def local_bounds(nodes: np.ndarray, roots: np.ndarray) -> np.ndarray:
    """BLAS root boxes as f32 (the reference's localBounds after a build/refit)."""
    return nodes[roots.astype(np.int64), 0:6].view(np.float32).copy()


def compute_tail(pool, materials: np.ndarray | None = None, nodes: np.ndarray | None = None):
    """computeDynamic + buildTlasRecords + writeDynamic (spectral_scene.js:1256-1366).

    Returns (materials with instance records and TLAS, order, liveInstanceBounds, aabbs)."""
    lib = load()
    n = pool.instCount
    nodes = pool.bvhNodes if nodes is None else nodes
    lb = np.ascontiguousarray(local_bounds(nodes, pool.inst_root))
    inv = np.zeros((n, 12), np.float32)
    det = np.zeros(n, np.float32)
    aabb = np.zeros((n, 9), np.float64)
    world = np.ascontiguousarray(pool.inst_world)
    act = np.ascontiguousarray(pool.inst_active)
    lib.orc_compute_instances(_p(world), _p(act), _p(lb), n, _p(inv), _p(det), _p(aabb))
    tl = np.zeros((2 * n + 2, 12), np.float32)
    order = np.zeros(n, np.uint32)
    cnt = lib.orc_build_tlas(_p(aabb), n, _p(tl), _p(order), None)
    assert cnt == pool.tlasNodeCount, (cnt, pool.tlasNodeCount)
    mats = (pool.materials if materials is None else materials).copy()
    ib = pool.instBase
    live = np.zeros((n, 6), np.float32)
    for slot in range(n):
        src = order[slot]
        r = np.zeros(28, np.float32)
        r[0:12] = inv[src]
        r[12] = pool.inst_root[src]
        r[13] = pool.inst_end[src]
        r[14] = det[src]
        r[15] = pool.inst_active[src]
        mats[ib + slot * 28: ib + slot * 28 + 28] = r
        live[slot] = aabb[src, 0:6].astype(np.float32)
    mats[pool.tlasBase: pool.tlasBase + cnt * 12] = tl[:cnt].reshape(-1)
    return mats, order, live, aabb


def scene_struct(pool, materials: np.ndarray, nodes: np.ndarray | None = None, vertex: np.ndarray | None = None,
                 keep=None) -> OrcScene:
    nodes = pool.bvhNodes if nodes is None else nodes
    vertex = pool.vertexData if vertex is None else vertex
    s = OrcScene()
    s.nodes = _p(nodes); s.nodeCount = nodes.shape[0]
    s.triIndex = _p(pool.triIndex); s.triCount = pool.triIndex.shape[0]
    s.vertexData = _p(vertex); s.vertexCount = vertex.shape[0]
    s.triMaterial = _p(pool.triMaterial)
    s.materials = _p(materials); s.materialsLen = materials.shape[0]
    s.instBase = pool.instBase; s.instCount = pool.instCount
    s.tlasBase = pool.tlasBase; s.tlasNodeCount = pool.tlasNodeCount
    if keep is not None:
        keep.extend([nodes, vertex, materials, pool.triIndex, pool.triMaterial])
    return s


def grid_struct(g: dict) -> OrcGrid:
    o = OrcGrid()
    gs = np.asarray(g["gridSize"], np.float32).astype(np.float64)
    gm = np.asarray(g["gridMin"], np.float32).astype(np.float64)
    res = g["res"]
    for a in range(3):
        o.gridMin[a] = gm[a]; o.gridSize[a] = gs[a]; o.res[a] = res[a]
    o.rays = g["rays"]
    o.maxDist = float(np.float32(g["maxDist"]))
    o.cellMin = float(np.float32(g["cellMin"]))
    return o


def light_arena(records: np.ndarray, clustered: bool, grid0: dict | None) -> np.ndarray:
    """The fixed 64x17 record arena, plus the C0 cell lists when clustered
    (lightGridKernel evaluated in FP32)."""
    lib = load()
    cells = 0
    if clustered:
        r = grid0["res"]
        cells = (r[0] - 1) * (r[1] - 1) * (r[2] - 1)
    arena = np.zeros(64 * 17 + cells * 17, np.float32)
    recs = np.asarray(records, np.float32).reshape(-1, 17)
    arena[:recs.size] = recs.reshape(-1)
    if clustered:
        g = grid_struct(grid0)
        lib.orc_light_grid(C.byref(g), _p(arena), recs.shape[0], _p(arena), 1)
    return arena


def solve(scene: OrcScene, arena: np.ndarray, light_count: int, clustered: bool, grid: OrcGrid, grid0: OrcGrid,
          params: np.ndarray, probe_offset: int, updated: int, irr: np.ndarray, depth: np.ndarray,
          atlas: np.ndarray, depth_atlas: np.ndarray, fp32: bool = False, io: OrcSolveIO | None = None,
          nthreads: int | None = None, emitters: tuple = (0, 0)) -> None:
    """One solve; `emitters` = (emitterBase, emitterCount) of the arena's
    giEmitter records, whose visibility history lives in io.emitterVis."""
    lib = load()
    L = OrcLights()
    L.data = _p(arena); L.dataLen = arena.shape[0]; L.lightCount = light_count; L.clustered = 1 if clustered else 0
    L.emitterBase, L.emitterCount = int(emitters[0]), int(emitters[1])
    prm = np.ascontiguousarray(params, np.float64)
    assert prm.shape[0] == lib.orc_params_size()
    f = lib.orc_solve_f32 if fp32 else lib.orc_solve_f64
    rc = f(C.byref(scene), C.byref(L), C.byref(grid), C.byref(grid0), _p(prm), probe_offset, updated, _p(irr),
           _p(depth), _p(atlas), _p(depth_atlas), C.byref(io) if io is not None else None,
           nthreads or threads())
    assert rc == 0


def new_state(grid: dict, fp32: bool = False):
    r = grid["res"]
    P = r[0] * r[1] * r[2]
    dt = np.float32 if fp32 else np.float64
    W, H = r[0] * 8, r[1] * r[2] * 8
    atlas = np.zeros((H, W, 4), np.uint16)
    atlas[..., 3] = 0x3C00  # (0,0,0,1), clearAtlasKernel
    return (np.zeros(P * 64 * 4, dt), np.zeros(P * 64 * 2, dt), atlas, atlas.copy())


REFLECT_TIERS = {"off": 0, "rough": 1, "high": 2, "ultra": 3}


class ReflectState:
    """The oracle's reflection lobe state of one cascade for a tier (1 rough,
    2 high, 3 ultra; REFLECTION_QUALITY_TIERS, gi_probes.js:60-75): the rough
    history and atlas in the irradiance layout, and for high / ultra the
    glossy numerator, support and atlas (tiles of glossyOct + 2 texels packed
    ceil(sqrt(probes)) to a row, gi_probes.js:3103-3110) and the glossy phase."""

    def __init__(self, grid: dict, tier: int, fp32: bool = False):
        r = grid["res"]
        P = r[0] * r[1] * r[2]
        dt = np.float32 if fp32 else np.float64
        self.tier = int(tier)
        self.rough = np.zeros(P * 64 * 4, dt)
        self.rough_atlas = np.zeros((r[1] * r[2] * 8, r[0] * 8, 4), np.uint16)
        self.oct = 8 if tier == 2 else 16 if tier == 3 else 1
        self.tile = self.oct + 2 if tier >= 2 else 1
        self.interval = 2 if tier == 2 else 1 if tier == 3 else 0
        self.tiles_x = max(1, math.ceil(math.sqrt(P))) if tier >= 2 else 1
        self.tiles_y = max(1, -(-P // self.tiles_x)) if tier >= 2 else 1
        self.glossy_num = np.zeros(P * self.tile * self.tile * 4, dt)
        self.glossy_den = np.zeros(P * self.tile * self.tile, dt)
        self.glossy_atlas = np.zeros((self.tiles_y * self.tile, self.tiles_x * self.tile, 4), np.uint16)
        self.phase = 0

    def attach(self, io: OrcSolveIO) -> None:
        io.reflectTier, io.glossyPhase = self.tier, self.phase
        io.roughSpec, io.roughAtlas = _p(self.rough), _p(self.rough_atlas)
        io.glossyNum, io.glossyDen, io.glossyAtlas = _p(self.glossy_num), _p(self.glossy_den), _p(self.glossy_atlas)

    def advance(self) -> None:
        """After a solve: the next solve resolves the next glossy phase."""
        if self.interval:
            self.phase = (self.phase + 1) % self.interval


def adjoint(scene: OrcScene, arena: np.ndarray, light_count: int, clustered: bool, grid: OrcGrid,
            params: np.ndarray, tri: np.ndarray, inst: np.ndarray, blocked: np.ndarray, solves: int,
            albedo: np.ndarray, emissive: np.ndarray, light_scale: np.ndarray, target: np.ndarray | None = None,
            round_atlas: bool = True, grad: bool = True, nthreads: int | None = None):
    """FP64 differentiable solve sequence (orc_adjoint.hpp).

    Replays fixed per-ray hit records (tri, inst | facing << 31) and blocked
    shadow bits for every solve. Returns (loss, E[probes*36*3], grad or None)
    with grad = [albedo (mc*3) | emissive (mc*3) | light scale (lights)]."""
    lib = load()
    if not hasattr(lib, "_adj"):
        P = C.c_void_p
        lib.orc_adjoint.restype = C.c_int
        lib.orc_adjoint.argtypes = [P, P, P, P, P, P, P, C.c_uint32, C.c_int32, P, P, P, C.c_uint32, C.c_uint32,
                                    P, P, P, P, C.c_int32]
        lib._adj = True
    L = OrcLights()
    L.data = _p(arena); L.dataLen = arena.shape[0]; L.lightCount = light_count; L.clustered = 1 if clustered else 0
    prm = np.ascontiguousarray(params, np.float64)
    mc = albedo.size // 3
    alb = np.ascontiguousarray(albedo, np.float64)
    emi = np.ascontiguousarray(emissive, np.float64)
    ls = np.ascontiguousarray(light_scale, np.float64)
    tri = np.ascontiguousarray(tri, np.int32)
    inst = np.ascontiguousarray(inst, np.int32)
    blocked = np.ascontiguousarray(blocked, np.uint64)
    probes = grid.res[0] * grid.res[1] * grid.res[2]
    E = np.zeros(probes * 36 * 3, np.float64)
    loss = C.c_double(0.0)
    tgt = None if target is None else np.ascontiguousarray(target, np.float64)
    g = np.zeros(6 * mc + ls.size, np.float64) if (grad and tgt is not None) else None
    rc = lib.orc_adjoint(C.byref(scene), C.byref(L), C.byref(grid), _p(prm), _p(tri), _p(inst), _p(blocked),
                         solves, 1 if round_atlas else 0, _p(alb), _p(emi), _p(ls), mc, ls.size, _p(tgt),
                         C.byref(loss), _p(E), _p(g), nthreads or threads())
    assert rc == 0
    return loss.value, E, g


# ------------------------------------------------- hit-ID disagreement proof
HIT_CODES = {0: "same", 1: "near-tie", 2: "gpu edge graze", 3: "oracle edge graze", 4: "t order within FP32 error",
             5: "unexplained"}


def probe_rays(grid: OrcGrid, jitter: float, probe_offset: int, updated: int):
    """FP64 world-space probe rays of a solve (origin, direction per ray)."""
    n = updated * grid.rays
    ro = np.zeros((n, 3), np.float64)
    rd = np.zeros((n, 3), np.float64)
    load().orc_probe_rays(C.byref(grid), float(jitter), probe_offset, updated, _p(ro), _p(rd))
    return ro, rd


def explain_hits(scene: OrcScene, ro: np.ndarray, rd: np.ndarray, g_tri, g_inst, o_tri, o_inst, o_t):
    """Per ray, why the GPU's closest hit (g_tri, g_inst) differs from the FP64
    oracle's (o_tri, o_inst, o_t): a code of HIT_CODES, plus the FP64 t of the
    GPU's pair (-1 when it has none)."""
    n = ro.shape[0]
    ro = np.ascontiguousarray(ro, np.float64)
    rd = np.ascontiguousarray(rd, np.float64)
    arrs = [np.ascontiguousarray(a, np.int32) for a in (g_tri, g_inst, o_tri, o_inst)]
    ot = np.ascontiguousarray(o_t, np.float64)
    code = np.zeros(n, np.int32)
    gt = np.zeros(n, np.float64)
    load().orc_explain_hits(C.byref(scene), _p(ro), _p(rd), n, *[_p(a) for a in arrs], _p(ot), _p(code), _p(gt),
                            threads())
    return code, gt


def pair_t(scene: OrcScene, ro: np.ndarray, rd: np.ndarray, tri, inst) -> np.ndarray:
    """FP64 t of each ray's (tri, inst) pair on that ray (-1 without a pair)."""
    n = ro.shape[0]
    out = np.zeros(n, np.float64)
    load().orc_pair_t(C.byref(scene), _p(np.ascontiguousarray(ro, np.float64)), _p(np.ascontiguousarray(rd, np.float64)),
                      n, _p(np.ascontiguousarray(tri, np.int32)), _p(np.ascontiguousarray(inst, np.int32)), _p(out),
                      threads())
    return out


# ----------------------------------------------------- per-tick scheduling
class Schedule:
    """The reference's per-tick solve schedule for one cascade: probes per tick
    (updatedCap / tickCap, gi_probes.js:2947-2962), the round-robin cursor and
    the per-cascade service-interval EMA and hysteresis exponent (3737-3766,
    3788, 3838-3839; probeUpdateIntervalTicks 197-202,
    hysteresisExponentForInterval 235-251), and the montecarlo jitter epoch
    (3776-3787). One C0 cascade, the fallback service interval of one tick."""

    DT_REF_MS = 1000.0 / 60.0

    def __init__(self, probe_total: int, rays: int, ray_budget: int, max_probes: int, montecarlo: bool,
                 normalize: bool):
        self.total = probe_total
        self.rays = rays
        self.cap = max(1, min(max_probes, ray_budget // max(1, rays)))
        self.montecarlo = montecarlo
        self.normalize = normalize
        self.cursor = 0
        self.last = 0.0
        self.ema = 0.0
        self.frame = 0
        self.jitter = 0.0

    def tick(self, now_ms: float) -> dict:
        updated = min(self.cap, self.total)
        ema = self.ema
        if self.last > 0:
            dt = now_ms - self.last
            ema = (ema * 0.8 + dt * 0.2 if ema > 0 else dt) if 0 < dt < 200 else 0.0
        service = ema if ema > 0 else self.DT_REF_MS
        revisit = max(1.0, self.total / max(1, updated))
        exponent = load().orc_hysteresis_exponent(service * revisit, 1 if self.normalize else 0)
        if self.montecarlo:
            self.frame = (self.frame + 1) & 0xFFFFFFFF
            self.jitter = (self.frame * 0.61803398875) % 1
        out = dict(probeOffset=self.cursor, updatedCount=updated, hysteresisExponent=exponent, frameJitter=self.jitter)
        self.cursor = (self.cursor + updated) % self.total if self.total else 0
        self.last = now_ms
        self.ema = ema
        return out


# --------------------------------------------- scene pool on the oracle side
# The reference arm of the benchmark and the pool cross-check build their
# scene with these restatements only, never with the CUDA library's host code.

ORC_PARAM_NAMES = [
    "frameJitter", "emitterVisSeed", "hysteresis", "hysteresisExponent",
    "depthSharpness", "radianceClamp", "classifyStrength", "filterStrength", "filterSmooth",
    "tempChangeSigma1", "tempChangeHDrop", "tempClampSigma", "nirGate", "nirGain", "skyIntensity",
] + [f"skySH{i}" for i in range(27)] + [
    "debugTraceBiasScale", "debugRayEpsScale", "debugDirectScale", "debugEmissiveScale",
    "debugAlbedoScale", "debugBounceScale", "debugCosinePower",
    "debugTempNoiseHBoost", "debugTempChangeSigma0", "debugTempMinChangeH",
    "debugTempVarEps", "debugTempVarRel", "debugDepthHistoryScale",
    "debugFilterKScale", "debugFilterRelScale", "debugFilterEpsScale",
    "reflectionSkyFallback", "skyConfigured",
]


def default_params(hysteresis: float = 0.60) -> np.ndarray:
    """The shared uniforms `U` at their initial values (gi_probes.js:1198-1255;
    temporal constants 182-189; JITTER_HYSTERESIS_DEFAULTS.gated = 0.60), in the
    order of the oracle's Params, each rounded to float32 as a uniform stores it."""
    v = dict.fromkeys(ORC_PARAM_NAMES, 0.0)
    v.update(hysteresis=hysteresis, hysteresisExponent=1.0, depthSharpness=7.0, radianceClamp=8.0,
             filterStrength=1.0, filterSmooth=0.5, tempChangeSigma1=2.5, tempChangeHDrop=0.30, tempClampSigma=6.0,
             nirGain=1.0, skyIntensity=1.0, debugTraceBiasScale=1.0, debugRayEpsScale=1.0, debugDirectScale=1.0,
             debugEmissiveScale=1.0, debugAlbedoScale=1.0, debugBounceScale=1.0, debugCosinePower=1.0,
             debugTempNoiseHBoost=0.25, debugTempChangeSigma0=0.75, debugTempMinChangeH=0.55,
             debugTempVarEps=0.000025, debugTempVarRel=0.0025, debugDepthHistoryScale=1.0, debugFilterKScale=1.0,
             debugFilterRelScale=1.0, debugFilterEpsScale=1.0)
    out = np.array([np.float32(v[n]) for n in ORC_PARAM_NAMES], np.float64)
    assert out.shape[0] == load().orc_params_size()
    return out


def select_light_records(records: np.ndarray, importance_ranked: bool, grid_min, grid_max):
    """selectGiLightRecords / selectGiLights / giLightImportance
    (gi_probes.js:4253-4289): analytic records (type < 2.5) first, importance
    top-K by (score desc, index asc) when clustered, then up to 16 emitters.
    Returns (records, analytic count, emitter count)."""
    recs = [np.asarray(r, np.float32) for r in np.asarray(records, np.float32).reshape(-1, 17)]
    analytic = [r for r in recs if abs(float(r[0]) - 3) >= 0.5 and float(r[0]) < 2.5]
    emitters = [r for r in recs if abs(float(r[0]) - 3) < 0.5]
    n_emit = min(16, len(emitters))
    budget = 64 - n_emit

    def score(r):
        if r[0] < 0.5:
            return float("inf")
        power = max(float(r[7]), float(r[8]), float(r[9]))
        cone = max(0.02, (1 - float(r[12])) * 0.5) if abs(float(r[0]) - 2) < 0.5 else 1.0
        d = [max(grid_min[a] - float(r[1 + a]), 0.0, float(r[1 + a]) - grid_max[a]) for a in range(3)]
        return (power * cone) / (1 + d[0] * d[0] + d[1] * d[1] + d[2] * d[2])

    if importance_ranked and len(analytic) > budget:
        keep = sorted(range(len(analytic)), key=lambda i: (-score(analytic[i]), i))[:budget]
        analytic = [analytic[i] for i in keep]
    else:
        analytic = analytic[:budget]
    out = analytic + emitters[:n_emit]
    arr = np.stack(out) if out else np.zeros((0, 17), np.float32)
    return arr, len(analytic), n_emit


def build_blas(positions: np.ndarray, indices: np.ndarray, leaf: int = 8):
    """MeshBVH + flattenBVHRoot of one mesh (orc_bvh.hpp): (nodes (N,8) u32,
    triangle order, index triples in BVH order)."""
    lib = load()
    if not hasattr(lib, "_bvh"):
        P = C.c_void_p
        lib.orc_build_blas.restype = C.c_uint32
        lib.orc_build_blas.argtypes = [P, C.c_uint32, P, C.c_uint32, C.c_uint32, P, C.c_uint64, P]
        lib._bvh = True
    pos = np.ascontiguousarray(positions, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32).copy()
    T = idx.shape[0]
    nodes = np.zeros((2 * T + 1, 8), np.uint32)
    order = np.zeros(T, np.uint32)
    n = lib.orc_build_blas(_p(pos), pos.shape[0], _p(idx), T, leaf, _p(nodes), nodes.shape[0], _p(order))
    if n == 0:
        raise ValueError("BLAS build failed (empty mesh, out-of-range index or oversized leaf)")
    return nodes[:n].copy(), order, idx


def tlas_node_count(n: int) -> int:
    """Records of buildTlasRecords' median split with leaves of <= 2 instances
    (spectral_scene.js:973-1003)."""
    t = [1] * (n + 1)
    for m in range(3, n + 1):
        t[m] = 1 + t[m >> 1] + t[m - (m >> 1)]
    return t[n] if n else 0


class OrcPool:
    """The typed arrays of buildSpectralScene for a plain mesh scene: pooled
    BLASes with pool-absolute miss links and leaf offsets (spectral_scene.js:
    1188-1240), the material records followed by room for the instance records
    and the TLAS (1327-1334), and the instance table (column-major FP64 world
    matrices, three's Matrix4.elements)."""

    def __init__(self, scene, leaf: int = 8):
        blas = [build_blas(m.positions, m.indices, leaf) for m in scene.meshes]
        nV = sum(m.positions.shape[0] for m in scene.meshes)
        nT = sum(m.indices.shape[0] for m in scene.meshes)
        nN = sum(b[0].shape[0] for b in blas)
        if nT >= 1 << 24 or nN >= 1 << 24:
            raise ValueError("BVH pool exceeds the 24-bit index ceiling")
        self.vertexData = np.zeros((nV, 8), np.float32)
        self.triIndex = np.zeros((nT, 3), np.uint32)
        self.triMaterial = np.zeros(nT, np.uint32)
        self.bvhNodes = np.zeros((nN, 8), np.uint32)
        M = len(scene.meshes)
        self.blas_root = np.zeros(M, np.uint32); self.blas_end = np.zeros(M, np.uint32)
        self.vert_base = np.zeros(M, np.uint32); self.vert_count = np.zeros(M, np.uint32)
        v0 = t0 = n0 = 0
        for i, (mesh, (nodes, order, idx)) in enumerate(zip(scene.meshes, blas)):
            V, T, N = mesh.positions.shape[0], idx.shape[0], nodes.shape[0]
            self.vertexData[v0:v0 + V, 0:3] = mesh.positions
            if mesh.normals is not None:
                self.vertexData[v0:v0 + V, 3:6] = mesh.normals
            if mesh.uvs is not None:
                self.vertexData[v0:v0 + V, 6:8] = mesh.uvs
            self.triIndex[t0:t0 + T] = idx + v0
            self.triMaterial[t0:t0 + T] = np.asarray(mesh.tri_material, np.uint32)[order]
            b = nodes.copy()
            b[:, 6] += n0
            lf = b[:, 7] != 0xFFFFFFFF
            b[lf, 7] = (b[lf, 7] & 0xFF000000) | (((b[lf, 7] & 0x00FFFFFF) + t0) & 0x00FFFFFF)
            self.bvhNodes[n0:n0 + N] = b
            self.blas_root[i], self.blas_end[i] = n0, n0 + N
            self.vert_base[i], self.vert_count[i] = v0, V
            v0 += V; t0 += T; n0 += N
        ubers = np.asarray(scene.materials, np.float32).reshape(-1, 28)
        I = len(scene.instances)
        self.instCount = I
        self.tlasNodeCount = tlas_node_count(I)
        self.instBase = ubers.shape[0] * 28
        self.tlasBase = self.instBase + I * 28
        self.materials = np.zeros(self.tlasBase + self.tlasNodeCount * 12, np.float32)
        self.materials[:self.instBase] = ubers.reshape(-1)
        self.inst_world = np.zeros((I, 16), np.float64)
        self.inst_active = np.zeros(I, np.uint8)
        self.inst_root = np.zeros(I, np.uint32); self.inst_end = np.zeros(I, np.uint32)
        for k, inst in enumerate(scene.instances):
            self.inst_world[k] = np.asarray(inst.world, np.float64).T.reshape(16)
            self.inst_active[k] = 1 if inst.active else 0
            self.inst_root[k] = self.blas_root[inst.mesh]
            self.inst_end[k] = self.blas_end[inst.mesh]


def grid_dict(grid_min, grid_size, res, rays) -> dict:
    """A cascade's grid uniforms (makeCascadeU, gi_probes.js:1010-1024): maxDist =
    |gridSize|, cellMin = the smallest probe spacing (floor 1e-4)."""
    gs = np.asarray(grid_size, np.float64)
    return dict(gridMin=list(grid_min), gridSize=list(grid_size), res=list(res), rays=rays,
                maxDist=float(np.linalg.norm(gs)),
                cellMin=float(max(1e-4, min(gs[a] / max(1, res[a] - 1) for a in range(3)))))



# ---------------------------------------------------------- receiver gather
GATHER_PARAM_NAMES = ["normalBias0", "normalBias1", "chebyBias0", "chebyBias1", "chebyStrength", "detailStrength",
                      "intensity", "enabled", "samplePositionScale", "sampleBiasScale", "borderBand", "cascades",
                      "dualDetail", "reflectionIntensity", "roughnessLimit"]


def gather_params(**kw) -> np.ndarray:
    """The receiver's uniforms at their initial values (gi_probes.js:314-358:
    normalBias 0.04, chebyBias 0, detailStrength 1, intensity 1, chebyStrength
    0, borderBand 0.15, the sample scales 1, one cascade), overridden by `kw`,
    each rounded to float32 as a uniform stores it."""
    v = dict(normalBias0=0.04, normalBias1=0.04, chebyBias0=0.0, chebyBias1=0.0, chebyStrength=0.0,
             detailStrength=1.0, intensity=1.0, enabled=1.0, samplePositionScale=1.0, sampleBiasScale=1.0,
             borderBand=0.15, cascades=1.0, dualDetail=0.0, reflectionIntensity=1.0, roughnessLimit=1.0)
    v.update(kw)
    out = np.array([np.float32(v[k]) for k in GATHER_PARAM_NAMES], np.float64)
    assert out.shape[0] == load().orc_gather_params_size()
    return out


def gather(grid0: OrcGrid, atlas0: np.ndarray, depth0: np.ndarray, params: np.ndarray, pos4: np.ndarray,
           nvis4: np.ndarray, ndir4: np.ndarray, grid1: OrcGrid | None = None, atlas1: np.ndarray | None = None,
           depth1: np.ndarray | None = None):
    """FP64 receiver irradiance at n surface points (n x 3) and each point's
    distance to a discontinuity of the gather (cage floor, Chebyshev select)."""
    n = pos4.shape[0]
    out = np.zeros((n, 3), np.float64)
    near = np.zeros(n, np.float64)
    arr = [np.ascontiguousarray(a, np.float32) for a in (pos4, nvis4, ndir4)]
    load().orc_gather(C.byref(grid0), C.byref(grid1) if grid1 is not None else None, _p(atlas0), _p(depth0),
                      _p(atlas1), _p(depth1), _p(np.ascontiguousarray(params, np.float64)), *[_p(a) for a in arr], n,
                      _p(out), _p(near), threads())
    return out, near


class OrcReflectAtlas(C.Structure):
    _fields_ = [("rough", C.c_void_p), ("glossy", C.c_void_p), ("glossyOct", C.c_uint32), ("glossyTile", C.c_uint32),
                ("glossyTilesX", C.c_uint32), ("glossyW", C.c_uint32), ("glossyH", C.c_uint32)]


def reflect_atlas(rough: np.ndarray, glossy: np.ndarray | None = None, oct_: int = 0, tiles_x: int = 1):
    """A cascade's reflection atlases for gather_combined: the rough atlas (H x
    W x 4 binary16) and, for tiers high / ultra, the glossy atlas with its
    octahedral resolution and tiles per row."""
    r = OrcReflectAtlas()
    r.rough = _p(rough)
    r._keep = (rough, glossy)
    if glossy is not None:
        r.glossy = _p(glossy)
        r.glossyOct, r.glossyTile, r.glossyTilesX = oct_, oct_ + 2, tiles_x
        r.glossyH, r.glossyW = glossy.shape[0], glossy.shape[1]
    return r


def gather_combined(grid0: OrcGrid, atlas0, depth0, refl0: OrcReflectAtlas, params: np.ndarray, pos4, nvis4, ndir4,
                    rdir4, grid1: OrcGrid | None = None, atlas1=None, depth1=None,
                    refl1: OrcReflectAtlas | None = None):
    """FP64 combined receiver at n points: irradiance (n x 3), the reflection
    layer (n x 4: rgb x weight, coverage x weight) and each point's distance to
    a discontinuity (cage floor, Chebyshev select, parallax root selects,
    roughness limit)."""
    lib = load()
    if not hasattr(lib, "_gc"):
        P = C.c_void_p
        lib.orc_gather_combined.restype = None
        lib.orc_gather_combined.argtypes = [P] * 13 + [C.c_uint32, P, P, P, C.c_int32]
        lib._gc = True
    n = pos4.shape[0]
    irr = np.zeros((n, 3), np.float64)
    refl = np.zeros((n, 4), np.float64)
    near = np.zeros(n, np.float64)
    arr = [np.ascontiguousarray(a, np.float32) for a in (pos4, nvis4, ndir4, rdir4)]
    lib.orc_gather_combined(C.byref(grid0), C.byref(grid1) if grid1 is not None else None, _p(atlas0), _p(depth0),
                            _p(atlas1), _p(depth1), C.byref(refl0), C.byref(refl1) if refl1 is not None else None,
                            _p(np.ascontiguousarray(params, np.float64)), *[_p(a) for a in arr], n, _p(irr), _p(refl),
                            _p(near), threads())
    return irr, refl, near


# ------------------------------------------------- fine cascade placement
def js_to_int32(x: np.ndarray) -> np.ndarray:
    """ECMAScript ToInt32 (the `| 0` operator) of float64 values."""
    x = np.asarray(x, np.float64)
    out = np.zeros(x.shape, np.int64)
    fin = np.isfinite(x)
    t = np.trunc(x[fin])
    m = np.fmod(t, 4294967296.0)
    m = np.where(m < 0, m + 4294967296.0, m)
    m = np.where(m >= 2147483648.0, m - 4294967296.0, m)
    out[fin] = m.astype(np.int64)
    return out


def fit_fine_box(vertex_data: np.ndarray, tri_index: np.ndarray, box_min, box_size):
    """fitFineBox (gi_probes.js:2968-3030) in float64, JS semantics: 16^3
    histogram of the pooled triangles' centroids ((v0 + v1 + v2) / 3 of the
    pooled vertexData), bins >= 0.4 x peak united, padded by one bin, each
    axis clamped to [0.25, 0.60] of the box and slid inside it. Returns
    (min[3], size[3]) or None."""
    G = 16
    mn = [float(v) for v in box_min]
    size = [float(v) for v in box_size]
    inv = [G / max(1e-6, size[a]) for a in range(3)]
    vd = np.asarray(vertex_data, np.float32).reshape(-1, 8)[:, 0:3].astype(np.float64)
    ti = np.asarray(tri_index, np.int64).reshape(-1, 3)
    c = ((vd[ti[:, 0]] + vd[ti[:, 1]]) + vd[ti[:, 2]]) / 3.0
    g = [np.clip(js_to_int32((c[:, a] - mn[a]) * inv[a]), 0, G - 1) for a in range(3)]
    hist = np.bincount((g[2] * G + g[1]) * G + g[0], minlength=G ** 3)
    peak = int(hist.max()) if hist.size else 0
    if peak == 0:
        return None
    thr = peak * 0.4
    sel = np.flatnonzero(hist >= thr)
    if sel.size == 0:
        return None
    xs, ys, zs = sel % G, (sel // G) % G, sel // (G * G)
    bx0, bx1, by0, by1, bz0, bz1 = int(xs.min()), int(xs.max()), int(ys.min()), int(ys.max()), int(zs.min()), int(zs.max())
    if bx0 == 0 and by0 == 0 and bz0 == 0 and bx1 == G - 1 and by1 == G - 1 and bz1 == G - 1:
        return None
    cell = [size[a] / G for a in range(3)]
    lo_b, hi_b = (bx0, by0, bz0), (bx1, by1, bz1)
    fmin = [mn[a] + lo_b[a] * cell[a] for a in range(3)]
    fmax = [mn[a] + (hi_b[a] + 1) * cell[a] for a in range(3)]
    pad = min(cell[0], cell[1], cell[2])
    fmin = [v - pad for v in fmin]
    fmax = [v + pad for v in fmax]
    fsize = [fmax[a] - fmin[a] for a in range(3)]
    box0max = [mn[a] + size[a] for a in range(3)]
    for a in range(3):
        lo, hi = 0.25 * size[a], 0.60 * size[a]
        s = max(lo, min(hi, fsize[a]))
        center = (fmin[a] + fmax[a]) * 0.5
        m0, m1 = center - s * 0.5, center + s * 0.5
        if m0 < mn[a]:
            m1 += (mn[a] - m0)
            m0 = mn[a]
        if m1 > box0max[a]:
            m0 -= (m1 - box0max[a])
            m1 = box0max[a]
        m0 = max(m0, mn[a])
        m1 = min(m1, box0max[a])
        fmin[a] = m0
        fsize[a] = max(1e-4, m1 - m0)
    return fmin, fsize


def js_round(x: float) -> int:
    """Math.round: floor(x + 0.5)."""
    return int(np.floor(x + 0.5))


def compute_grid_resolution(size, target_long_axis: int):
    """computeGridResolution (gi_probes.js:938-943)."""
    longest = max(size[0], size[1], size[2], 1e-3)
    spacing = longest / max(1, target_long_axis)
    return [int(min(32, max(2, js_round(s / spacing) + 1))) for s in size]


def fine_cascade_res(fine_size, target_long_axis: int, c0_probes: int):
    """C1's resolution (gi_probes.js:3396-3406): ~2x the coarse long-axis
    density, then shrunk by 0.85 per axis (at most 12 times) while above
    max(64, 2 x C0's probes)."""
    res = compute_grid_resolution(fine_size, min(32, js_round(target_long_axis * 2.0)))
    cap = max(64, 2 * c0_probes)
    for _ in range(12):
        if res[0] * res[1] * res[2] <= cap:
            break
        res = [max(2, int(np.floor(r * 0.85))) for r in res]
    return res


class Schedule2:
    """The per-tick schedule with a fine cascade (gi_probes.js:3581-3618,
    3715-3788): the solve list (both cascades when the tick budget covers
    their union, else one per tick in turn), per cascade the probe count,
    cursor, service-interval EMA and hysteresis exponent, the tick-interval EMA
    as the fallback service interval (x2 when the cascades alternate), and the
    montecarlo epoch advanced on ticks that solve C0."""

    DT_REF_MS = 1000.0 / 60.0

    def __init__(self, totals, rays: int, ray_budget: int, max_probes: int, montecarlo: bool, normalize: bool):
        self.totals = list(totals)
        self.cap = max(1, min(max_probes, ray_budget // max(1, rays)))
        self.montecarlo = montecarlo
        self.normalize = normalize
        n = len(self.totals)
        self.cursor, self.last, self.ema = [0] * n, [0.0] * n, [0.0] * n
        self.turn = 0
        self.frame = 0
        self.jitter = 0.0
        self.seed_counter = 0
        self.seed = 0.0
        self.last_tick = 0.0
        self.tick_ema = 0.0

    def tick(self, now_ms: float) -> list:
        if self.last_tick > 0:
            dt = now_ms - self.last_tick
            self.tick_ema = (self.tick_ema * 0.8 + dt * 0.2 if self.tick_ema > 0 else dt) if 0 < dt < 100 else 0.0
        self.last_tick = now_ms
        have_c1 = len(self.totals) > 1
        full = self.cap >= sum(self.totals)
        if not have_c1:
            lst = [0]
        elif full:
            lst = [0, 1]
        else:
            lst = [self.turn % 2]
            self.turn = (self.turn + 1) & 0xFFFFFFFF
        fallback_ticks = 1 if (not have_c1 or full) else 2
        out = []
        for ci in lst:
            total = self.totals[ci]
            updated = min(self.cap, total)
            ema = self.ema[ci]
            if self.last[ci] > 0:
                dt = now_ms - self.last[ci]
                ema = (ema * 0.8 + dt * 0.2 if ema > 0 else dt) if 0 < dt < 200 else 0.0
            service = ema if ema > 0 else (self.tick_ema if self.tick_ema > 0 else self.DT_REF_MS) * fallback_ticks
            revisit = max(1.0, total / max(1, updated))
            exponent = load().orc_hysteresis_exponent(service * revisit, 1 if self.normalize else 0)
            if ci == 0 and self.montecarlo:
                self.seed_counter = (self.seed_counter + 1) & 0xFFFFFFFF
                self.seed = (self.seed_counter * 0.61803398875) % 1
                self.frame = (self.frame + 1) & 0xFFFFFFFF
                self.jitter = (self.frame * 0.61803398875) % 1
            out.append(dict(cascade=ci, probeOffset=self.cursor[ci], updatedCount=updated,
                            hysteresisExponent=exponent, frameJitter=self.jitter, emitterVisSeed=self.seed))
            self.cursor[ci] = (self.cursor[ci] + updated) % total if total else 0
            self.last[ci] = now_ms
            self.ema[ci] = ema
        return out
