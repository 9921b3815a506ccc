"""Host mirror of the reference's probe-field facade, driving the CUDA library.

``createProbeField`` mirrors gi_probes.js:945-4846 and ``installSpeedballGI``
mirrors install.js:216-503 for the update path: the same entry names, option
names and defaults, the same per-tick scheduling (round-robin probe cursor,
ray budget, jitter epochs, hysteresis exponent; gi_probes.js:2947-2962,
3732-3840) and the same dirty lanes (``markTransformsDirty``,
``markDeformsDirty``, ``markMaterialValuesDirty``, ``markTopologyDirty``;
3869-3937). Scenes are ``speedball_b200.scene.SceneDesc`` instead of a three.js
scene; every device step goes through libspeedball_cuda.so.

Not mirrored (outside the update path): the raster lights node, the material
graph receiver, reflection lobes, probe classification/relocation, the
frame-pacing auto-throttle and the idle gate of structural rebuilds.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Callable

import numpy as np

from . import _abi
from .scene import SceneDesc, build_pool, column_major

TILE = 8
MAX_PROBES_PER_AXIS = 32
TARGET_PROBES_LONG_AXIS = 12
RAYS_PER_PROBE_DEFAULT = 64
RAYS_MIN, RAYS_MAX = 32, 256
RAYS_PER_TICK = 98_304
MAX_PROBES_PER_TICK = 2048
MAX_RAY_BUDGET = 524_288
MAX_LIGHTS = 64
GI_EMITTER_INJECT_CAP = 16
SURFACE_NORMAL_BIAS_CELL = 0.03
JITTER_HYSTERESIS_DEFAULTS = {"gated": 0.60, "montecarlo": 0.90}
HYSTERESIS_DT_REF_MS = 1000.0 / 60.0
TICK_OVERLOAD_MS = 100.0
C1_RES_SCALE = 2.0


REFLECTION_QUALITY_TIERS = ("off", "rough", "high", "ultra")


def resolveReflectionQuality(reflectionQuality=None, roughReflections=False) -> str:
    """resolveReflectionQuality (gi_probes.js:67-73): a tier name (off, rough,
    high, ultra; case and surrounding space ignored) or, when None, the legacy
    boolean (True = ultra, False = off)."""
    fallback = "ultra" if roughReflections is True else "off"
    name = fallback if reflectionQuality is None else str(reflectionQuality).strip().lower()
    if name not in REFLECTION_QUALITY_TIERS:
        raise ValueError(f'Unknown reflectionQuality "{reflectionQuality}". Expected off, rough, high, or ultra.')
    return name


def hysteresisExponentForInterval(updateDtMs: float, normalize: bool = True) -> float:
    """gi_probes.js:235-251."""
    if not normalize:
        return 1.0
    dt = max(0.0, updateDtMs) if math.isfinite(updateDtMs) else HYSTERESIS_DT_REF_MS
    return min(1.0, dt / HYSTERESIS_DT_REF_MS)


def probeUpdateIntervalTicks(probeTotal, probesPerTick, solveEveryTicks=1) -> float:
    """gi_probes.js:197-202."""
    total = max(0.0, float(probeTotal or 0))
    cap = max(1.0, float(probesPerTick or 1))
    schedule = max(1.0, float(solveEveryTicks or 1))
    return schedule * max(1.0, total / cap)


def computeGridResolution(size, targetLongAxis=TARGET_PROBES_LONG_AXIS):
    """gi_probes.js:938-943 (Math.round = floor(x + 0.5))."""
    longest = max(size[0], size[1], size[2], 1e-3)
    spacing = longest / max(1, targetLongAxis)
    return tuple(int(min(MAX_PROBES_PER_AXIS, max(2, math.floor(s / spacing + 0.5) + 1))) for s in size)


def _normalize_jitter_mode(mode) -> str:
    m = str(mode or "").lower().replace(" ", "").replace("_", "").replace("-", "")
    return "montecarlo" if m in ("montecarlo", "mc") else "gated"


def selectGiLightRecords(records: np.ndarray, importanceRanked: bool, gridMin=None, gridMax=None):
    """gi_probes.js:4262-4289: analytic records first (importance top-K when
    clustered), then the emitter suffix (type 3)."""
    recs = [np.asarray(r, np.float32) for r in np.asarray(records, np.float32).reshape(-1, 17)]
    analytic = [r for r in recs if r[0] < 2.5]
    emitters = [r for r in recs if abs(r[0] - 3) < 0.5]
    emitter_count = min(GI_EMITTER_INJECT_CAP, len(emitters))
    budget = MAX_LIGHTS - emitter_count
    if importanceRanked and len(analytic) > budget:
        def score(rec):
            if rec[0] < 0.5:
                return math.inf
            power = max(rec[7], rec[8], rec[9])
            cone = max(0.02, (1 - rec[12]) * 0.5) if abs(rec[0] - 2) < 0.5 else 1.0
            d = [max(gridMin[a] - rec[1 + a], 0.0, rec[1 + a] - gridMax[a]) for a in range(3)]
            return (power * cone) / (1 + d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
        ranked = sorted(range(len(analytic)), key=lambda i: (-score(analytic[i]), i))[:budget]
        selected = [analytic[i] for i in ranked]
    else:
        selected = analytic[:budget]
    out = selected + emitters[:emitter_count]
    arr = np.stack(out) if out else np.zeros((0, 17), np.float32)
    return arr, len(selected), emitter_count


# sb_set_scene_bvh_build_mode
SCENE_BVH_BUILD_MODES = {"blocking": 0, "background": 1}

class ProbeField:
    """createProbeField (gi_probes.js:945) over one scene and one GPU."""

    def __init__(self, scene: SceneDesc, *, intensity=1.0, hysteresis=None, jitterMode="gated", divisions=12,
                 rays=RAYS_PER_PROBE_DEFAULT, cascades=2, clusteredLighting=False, volumes=None, device=0,
                 recordHits=False, onRebuilt: Callable | None = None, variant: str | None = None,
                 blasBuilder: str = "host", reflectionQuality: str | None = None, roughReflections=False,
                 reflectionSkyFallback=False, sceneBvhBuild: str = "blocking"):
        self._lib = _abi.load(variant)
        self._reflection = resolveReflectionQuality(reflectionQuality, roughReflections)
        if blasBuilder not in ("host", "gpu"):
            raise ValueError("blasBuilder: 'host' or 'gpu'")
        if sceneBvhBuild not in SCENE_BVH_BUILD_MODES:
            raise ValueError("sceneBvhBuild: 'blocking' or 'background'")
        self._blasBuilder = blasBuilder
        self._scene = scene
        self._intensity = float(intensity)
        self._jitterMode = _normalize_jitter_mode(jitterMode)
        base_h = hysteresis if (hysteresis is not None and math.isfinite(hysteresis)) else \
            JITTER_HYSTERESIS_DEFAULTS[self._jitterMode]
        self._hysteresis = min(0.99, max(0.0, float(base_h)))
        self._targetLongAxis = int(min(MAX_PROBES_PER_AXIS, max(2, round(divisions) or TARGET_PROBES_LONG_AXIS)))
        self._rays = int(min(RAYS_MAX, max(RAYS_MIN, round(float(rays) / 16) * 16 or RAYS_PER_PROBE_DEFAULT)))
        # cascades=2 places the fine cascade C1 with fitFineBox at every rebuild
        self._cascades = 2 if int(cascades or 1) >= 2 else 1
        self._haveC1 = False
        self._c1Grid = None
        self._clustered = clusteredLighting is True or isinstance(clusteredLighting, dict)
        self._volumes = volumes
        self._rayBudget = RAYS_PER_TICK
        self._maxProbesPerTick = MAX_PROBES_PER_TICK
        self._hysteresisNormalize = True
        self._frameCounter = 0
        self._emitterVisSeedCounter = 0
        self._solveTurn = 0
        self._lastTickAt = 0.0
        self._hysteresisTickDtEma = 0.0
        # per cascade (C0, C1): round-robin cursor, last solve time, service-interval EMA
        self._cursor = [0, 0]
        self._lastSolveAt = [0.0, 0.0]
        self._solveDtEma = [0.0, 0.0]
        self._disposed = False
        self._onRebuilt = onRebuilt
        self._pendingTransforms: set[int] = set()
        self._pendingAllTransforms = False
        self._pendingDeform = False
        self._pendingMaterials: set[int] = set()
        self._pendingTopology = False
        self._deformVersions = {}
        self._extraCascades = {}  # extra cascade boxes (ci >= 1) configured by configureCascade
        self._params = _abi.default_params()
        self._params.hysteresis = self._hysteresis
        self._params.reflectionSkyFallback = 1.0 if reflectionSkyFallback is True else 0.0
        self._frameJitterOverride = None
        flags = _abi.SB_CTX_RECORD_HITS if recordHits else 0
        opts = _abi.sb_device_opts(device, flags)
        h = C.c_void_p()
        _abi.check(self._lib.sb_create(C.byref(opts), C.byref(h)))
        self._ctx = h
        self.stats = {"solves": 0, "refits": 0, "transformUpdates": 0, "rebuilds": 0}
        # structural: the reflection buffers of every cascade follow the tier
        self._ck(self._lib.sb_set_reflection_quality(h, _abi.REFLECT_TIERS[self._reflection]))
        self._ck(self._lib.sb_set_scene_bvh_build_mode(h, SCENE_BVH_BUILD_MODES[sceneBvhBuild]))
        self._rebuild()

    # ------------------------------------------------------------- plumbing
    def _ck(self, status):
        _abi.check(status, self._ctx)

    def _rebuild(self):
        """rebuild() (gi_probes.js:3269-3455): pool, upload, TLAS, grid fit, lights."""
        lib = self._lib
        self._pool = pool = build_pool(self._scene, self._ctx if self._blasBuilder == "gpu" else None, lib)
        self._ck(lib.sb_upload_scene(self._ctx, C.byref(pool.view())))
        self._ck(lib.sb_set_instances(self._ctx, pool.instCount, _abi.ptr(pool.inst_world),
                                      _abi.ptr(pool.inst_active), _abi.ptr(pool.inst_root), _abi.ptr(pool.inst_end)))
        self._ck(lib.sb_build_tlas(self._ctx))
        self._deformVersions = {i: self._version(m) for i, m in enumerate(self._scene.meshes)}
        self._fit_grid()
        self._upload_lights()
        self._ck(lib.sb_set_params(self._ctx, C.byref(self._params)))
        self._cursor = [0, 0]
        self._lastSolveAt = [0.0, 0.0]
        self._solveDtEma = [0.0, 0.0]
        self.stats["rebuilds"] += 1
        if self._onRebuilt:
            self._onRebuilt()

    @staticmethod
    def _version(mesh):
        """Identity of a mesh's position data (the attribute version of the reference,
        spectral_scene.js:1846-1861): the array object plus an explicit counter."""
        return (id(mesh.positions), getattr(mesh, "version", 0))

    def _scene_bounds(self):
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        for inst in self._scene.instances:
            if not inst.active:
                continue
            P = self._scene.meshes[inst.mesh].positions.astype(np.float64)
            W = inst.world
            Q = P @ W[:3, :3].T + W[:3, 3]
            lo = np.minimum(lo, Q.min(0))
            hi = np.maximum(hi, Q.max(0))
        return lo, hi

    def _fit_grid(self):
        """C0 placement (gi_probes.js:3341-3367): manual volume or padded scene bounds."""
        vol = self._volumes
        if vol:
            box_min = np.asarray(vol["gridMin"], np.float64)
            size = np.asarray(vol["gridSize"], np.float64)
            res = tuple(int(min(MAX_PROBES_PER_AXIS, max(2, round(r)))) for r in vol["res"]) if vol.get("res") \
                else computeGridResolution(size, self._targetLongAxis)
        else:
            lo, hi = self._scene_bounds()
            size = hi - lo
            pad = size * 0.06
            box_min = lo - pad
            size = size + 2 * pad
            res = computeGridResolution(size, self._targetLongAxis)
        g = _abi.sb_grid()
        for a in range(3):
            g.gridMin[a] = float(box_min[a])
            g.gridSize[a] = float(size[a])
            g.res[a] = int(res[a])
        g.raysPerProbe = self._rays
        gs = np.array([g.gridSize[a] for a in range(3)], np.float64)
        g.maxDist = float(np.linalg.norm(gs))
        g.cellMin = float(max(1e-4, min(gs[a] / max(1, res[a] - 1) for a in range(3))))
        self._grid = g
        self._res = res
        self._probeTotal = int(res[0] * res[1] * res[2])
        self._ck(self._lib.sb_configure_cascade(self._ctx, 0, C.byref(g)))
        self._haveC1 = False
        self._c0Box = ([float(v) for v in box_min], [float(v) for v in size])
        if self._cascades >= 2:
            self._place_fine_cascade(box_min, size)

    def _place_fine_cascade(self, box_min, size):
        """C1 dims (gi_probes.js:3386-3410): fitFineBox over C0's box, ~2x the
        coarse long-axis density, shrunk while above max(64, 2 x C0's probes).
        No fine box (empty or uniform histogram): one cascade this build."""
        mn = (C.c_double * 3)(*[float(v) for v in box_min])
        # Box3(min, min + size).getSize(): (min + size) - min in doubles
        sz = (C.c_double * 3)(*[float(box_min[a] + size[a]) - float(box_min[a]) for a in range(3)])
        omin, osize, found = (C.c_double * 3)(), (C.c_double * 3)(), C.c_int32(0)
        self._ck(self._lib.sb_fit_fine_box(self._ctx, mn, sz, omin, osize, C.byref(found)))
        if not found.value:
            return
        fsize = [osize[a] for a in range(3)]
        self._c1Box = ([omin[a] for a in range(3)], fsize, [sz[a] for a in range(3)])
        res = computeGridResolution(fsize, min(MAX_PROBES_PER_AXIS, math.floor(self._targetLongAxis * C1_RES_SCALE + 0.5)))
        cap = max(64, 2 * self._probeTotal)
        for _ in range(12):
            if res[0] * res[1] * res[2] <= cap:
                break
            res = tuple(max(2, math.floor(r * 0.85)) for r in res)
        g = _abi.sb_grid()
        for a in range(3):
            g.gridMin[a] = omin[a]
            g.gridSize[a] = fsize[a]
            g.res[a] = int(res[a])
        g.raysPerProbe = self._rays
        g.maxDist = float(np.linalg.norm(np.asarray(fsize, np.float64)))
        g.cellMin = float(max(1e-4, min(fsize[a] / max(1, res[a] - 1) for a in range(3))))
        self._ck(self._lib.sb_configure_cascade(self._ctx, 1, C.byref(g)))
        self._c1Grid = g
        self._c1Total = int(res[0] * res[1] * res[2])
        self._haveC1 = True

    def _upload_lights(self):
        gmin = [self._grid.gridMin[a] for a in range(3)]
        gmax = [self._grid.gridMin[a] + self._grid.gridSize[a] for a in range(3)]
        recs, analytic, emitters = selectGiLightRecords(self._scene.lights, self._clustered, gmin, gmax)
        recs = np.ascontiguousarray(recs, np.float32)
        self._lightCount = recs.shape[0]
        self._ck(self._lib.sb_upload_lights(self._ctx, _abi.ptr(recs) if recs.size else None, recs.shape[0],
                                            analytic, emitters, 1 if self._clustered else 0))

    # ------------------------------------------------------------ scheduling
    def updatedCap(self) -> int:
        """gi_probes.js:2947-2958."""
        return max(1, min(self._maxProbesPerTick, self._rayBudget // max(1, self._rays)))

    def tick(self, idleMs: float = math.inf, playing: bool = False, nowMs: float | None = None) -> dict:
        """One tick (gi_probes.js:3472-3849): dirty lanes, then the solves of
        this tick: C0, or with a fine cascade both cascades when the ray budget
        covers their union, else one cascade per tick in turn. Returns the
        first solve's frame with every solve under "solves"."""
        if self._disposed:
            return {}
        self._tick_clock(nowMs)
        if self._pendingTopology:
            self._pendingTopology = False
            self._rebuild()
        # the dirty lanes first: their refits are the tick's first GPU work, and the
        # solve planning below (host only) overlaps them
        self._refresh_lanes()
        lst = self._solve_list()
        fallback = 1 if (not self._haveC1 or len(lst) == 2) else 2
        if 0 in lst:
            self._advance_epoch()
        solves = []
        for ci in lst:
            s = self._plan_solve(ci, nowMs, fallback)
            self._params.hysteresisExponent = s["hysteresisExponent"]
            self._params.hysteresis = self._hysteresis
            self._ck(self._lib.sb_set_params(self._ctx, C.byref(self._params)))
            self._ck(self._lib.sb_solve(self._ctx, ci, s["probeOffset"], s["updatedCount"]))
            self._commit_solve(s, nowMs)
            solves.append(s)
        out = dict(solves[0])
        out["solves"] = solves
        return out

    def _tick_clock(self, nowMs):
        """The tick-interval EMA (gi_probes.js:3581-3618): the fallback service
        interval of a cascade that has none of its own yet."""
        if nowMs is None:
            return
        if self._lastTickAt > 0:
            dt = nowMs - self._lastTickAt
            ema = self._hysteresisTickDtEma
            self._hysteresisTickDtEma = (ema * 0.8 + dt * 0.2 if ema > 0 else dt) if 0 < dt < TICK_OVERLOAD_MS else 0.0
        self._lastTickAt = nowMs

    def _solve_list(self) -> list:
        """gi_probes.js:3715-3727."""
        if not self._haveC1:
            return [0]
        if self.updatedCap() >= self._probeTotal + self._c1Total:
            return [0, 1]
        ci = self._solveTurn % 2
        self._solveTurn = (self._solveTurn + 1) & 0xFFFFFFFF
        return [ci]

    def _advance_epoch(self):
        """Montecarlo: a new ray basis and emitter target on every C0 solve
        (gi_probes.js:3766-3787); gated keeps both."""
        if self._jitterMode == "montecarlo":
            self._emitterVisSeedCounter = (self._emitterVisSeedCounter + 1) & 0xFFFFFFFF
            self._params.emitterVisSeed = (self._emitterVisSeedCounter * 0.61803398875) % 1
            self._frameCounter = (self._frameCounter + 1) & 0xFFFFFFFF
            self._params.frameJitter = self._frameJitterOverride if self._frameJitterOverride is not None \
                else (self._frameCounter * 0.61803398875) % 1
        elif self._frameJitterOverride is not None:
            self._params.frameJitter = self._frameJitterOverride

    def _plan_solve(self, ci: int, nowMs, fallbackTicks: int) -> dict:
        """One cascade's probe range and hysteresis exponent (gi_probes.js:3737-3766)."""
        total = self.cascadeProbes(ci)
        updated = min(self.updatedCap(), total)
        ema = self._solveDtEma[ci]
        if nowMs is not None and self._lastSolveAt[ci] > 0:
            dt = nowMs - self._lastSolveAt[ci]
            ema = (ema * 0.8 + dt * 0.2 if ema > 0 else dt) if 0 < dt < 200 else 0.0
        serviceDt = ema if ema > 0 else \
            (self._hysteresisTickDtEma if self._hysteresisTickDtEma > 0 else HYSTERESIS_DT_REF_MS) * fallbackTicks
        revisit = probeUpdateIntervalTicks(total, updated)
        return {"cascade": ci, "probeOffset": self._cursor[ci], "updatedCount": updated,
                "hysteresisExponent": hysteresisExponentForInterval(serviceDt * revisit, self._hysteresisNormalize),
                "_ema": ema}

    def _commit_solve(self, s: dict, nowMs):
        ci, total = s["cascade"], self.cascadeProbes(s["cascade"])
        self._cursor[ci] = (self._cursor[ci] + s["updatedCount"]) % total if total else 0
        self._solveDtEma[ci] = s["_ema"]
        if nowMs is not None:
            self._lastSolveAt[ci] = nowMs
        self.stats["solves"] += 1

    def beginTick(self, nowMs: float | None = None) -> dict:
        """The part of a C0 tick ahead of its solve: dirty lanes, the solve's
        probe range and its uniforms (jitter epoch, hysteresis exponent). A
        batched frame (speedball_b200.batch) solves several fields' ranges in
        one launch between beginTick and endTick; a field with a fine cascade
        ticks through tick()."""
        lib = self._lib
        self._tick_clock(nowMs)
        if self._pendingTopology:
            self._pendingTopology = False
            self._rebuild()
        # the uniforms first (host work only), so that the solve is enqueued right
        # behind the dirty lanes while the GPU runs them
        s = self._plan_solve(0, nowMs, 1)
        self._advance_epoch()
        self._params.hysteresisExponent = s["hysteresisExponent"]
        self._ck(lib.sb_set_params(self._ctx, C.byref(self._params)))
        self._refresh_lanes()
        return s

    def endTick(self, frame: dict, nowMs: float | None = None) -> None:
        self._commit_solve(frame, nowMs)

    def configureCascade(self, ci: int, gridMin, gridSize, res, rays: int | None = None) -> None:
        """An extra cascade box of this field (ci >= 1), solved through
        speedball_b200.batch or sb_solve directly; cascade 0 stays the fitted one."""
        if ci < 1:
            raise ValueError("cascade 0 is the field's fitted grid")
        g = _abi.sb_grid()
        for a in range(3):
            g.gridMin[a] = float(gridMin[a])
            g.gridSize[a] = float(gridSize[a])
            g.res[a] = int(res[a])
        g.raysPerProbe = int(rays or self._rays)
        gs = np.array([g.gridSize[a] for a in range(3)], np.float64)
        g.maxDist = float(np.linalg.norm(gs))
        g.cellMin = float(max(1e-4, min(gs[a] / max(1, g.res[a] - 1) for a in range(3))))
        self._ck(self._lib.sb_configure_cascade(self._ctx, ci, C.byref(g)))
        self._extraCascades[ci] = g

    def cascadeGrid(self, ci: int):
        """The sb_grid cascade `ci` was configured with: C0, the fitted fine
        cascade C1, or a cascade set by configureCascade."""
        if ci == 0:
            return self._grid
        if ci == 1 and self._haveC1 and ci not in self._extraCascades:
            return self._c1Grid
        return self._extraCascades[ci]

    def cascadeProbes(self, ci: int) -> int:
        g = self.cascadeGrid(ci)
        return int(g.res[0] * g.res[1] * g.res[2])

    def hasFineCascade(self) -> bool:
        return self._haveC1

    def _refresh_lanes(self):
        lib = self._lib
        if self._pendingMaterials:
            ub = np.ascontiguousarray(self._scene.materials, np.float32).reshape(-1)
            for m in sorted(self._pendingMaterials):
                rec = np.ascontiguousarray(ub[m * 28:(m + 1) * 28])
                self._ck(lib.sb_upload_range(self._ctx, _abi.BUF["MATERIALS"], m * 28, 28, _abi.ptr(rec)))
            self._pendingMaterials.clear()
        moving = self._pendingAllTransforms or bool(self._pendingTransforms)
        deformed = []
        if self._pendingDeform:
            self._pendingDeform = False
            # with a transform lane in the same tick, one instance update carries both
            deformed = self.refreshDeforms(carryTlas=not moving)
        if moving:
            if self._pendingAllTransforms:
                idx = set(range(len(self._scene.instances)))
            else:
                idx = set(self._pendingTransforms)
                meshes = set(deformed)
                idx.update(i for i, inst in enumerate(self._scene.instances) if inst.mesh in meshes)
            self._pendingAllTransforms = False
            self._pendingTransforms.clear()
            self.refreshTransforms(sorted(idx))

    def refreshTransforms(self, instances):
        """refreshTransforms -> updateTransforms (gi_probes.js:4164-4179, spectral_scene.js:1402-1514)."""
        if not instances:
            return
        src = np.ascontiguousarray(np.asarray(instances, np.uint32))
        world = np.ascontiguousarray(np.stack([column_major(self._scene.instances[i].world) for i in instances]))
        self._ck(self._lib.sb_update_transforms(self._ctx, _abi.ptr(src), _abi.ptr(world), src.shape[0]))
        self.stats["transformUpdates"] += 1

    def refreshDeforms(self, meshes=None, carryTlas: bool = True):
        """refreshDeforms -> updateDeforms (gi_probes.js:4209-4234, spectral_scene.js:1831-1927):
        re-gather each deformed mesh's pooled vertices, refit its BLAS on the GPU,
        then carry the new root bounds into the TLAS (rewriteInstanceRows:false).
        carryTlas=False leaves that last step to a following refreshTransforms over
        the deformed meshes' instances (same bounds, one TLAS refit). Returns the
        indices of the meshes refit."""
        pool = self._pool
        if meshes is None:
            # same-topology deforms only: a mesh counts as changed when its positions
            # array was replaced or written since the last refresh
            changed = [i for i, m in enumerate(self._scene.meshes) if self._version(m) != self._deformVersions.get(i)]
        else:
            changed = list(meshes)
        n = 0
        for i in changed:
            m = self._scene.meshes[i]
            if m.positions.shape[0] != int(pool.vert_count[i]):
                raise _abi.SbError(_abi.SB_ERR_LAYOUT_VIOLATION, f"mesh {i}: vertex count changed (topology edit)")
            self._deformVersions[i] = self._version(m)
            # positions, and normals when the mesh has them; uv keeps its build-time
            # value (spectral_scene.js:1866-1900). The library copies both arrays
            # before it returns.
            pos = np.ascontiguousarray(m.positions, np.float32)
            nrm = None if m.normals is None else np.ascontiguousarray(m.normals, np.float32)
            self._ck(self._lib.sb_update_deform_xyz(self._ctx, int(pool.vert_base[i]), int(pool.vert_count[i]),
                                                    _abi.ptr(pos), None if nrm is None else _abi.ptr(nrm),
                                                    int(pool.blas_root[i]), int(pool.blas_end[i])))
            n += 1
        if n:
            if carryTlas:
                self._ck(self._lib.sb_update_transforms(self._ctx, None, None, 0))
            self.stats["refits"] += n
        return changed

    # ------------------------------------------------------------ dirty API
    def markTransformsDirty(self, target=None):
        """gi_probes.js:3869-3878: an instance index, {'object': i}, a list, or None for all."""
        if target is None:
            self._pendingAllTransforms = True
            return
        targets = target if isinstance(target, (list, tuple, set)) else [target]
        for t in targets:
            i = t.get("object", t.get("instanceIndex")) if isinstance(t, dict) else t
            if isinstance(i, (int, np.integer)) and 0 <= i < len(self._scene.instances):
                self._pendingTransforms.add(int(i))

    def markDeformsDirty(self):
        self._pendingDeform = True

    def markMaterialValuesDirty(self, targets=None):
        n = np.asarray(self._scene.materials).reshape(-1, 28).shape[0]
        if targets is None:
            self._pendingMaterials.update(range(n))
        else:
            for t in (targets if isinstance(targets, (list, tuple, set)) else [targets]):
                if 0 <= int(t) < n:
                    self._pendingMaterials.add(int(t))

    def markTopologyDirty(self):
        self._pendingTopology = True

    def notifySceneChange(self, change: dict | None = None):
        change = change or {}
        if change.get("topology"):
            self.markTopologyDirty()
        if change.get("transforms") is not None:
            self.markTransformsDirty(change.get("transforms") or None)
        if change.get("deforms"):
            self.markDeformsDirty()
        if change.get("materials") is not None:
            self.markMaterialValuesDirty(change.get("materials") or None)

    # -------------------------------------------------------------- setters
    def setHysteresis(self, h):
        self._hysteresis = min(0.99, max(0.0, float(h)))
        self._params.hysteresis = self._hysteresis

    def getHysteresis(self):
        return self._hysteresis

    def setHysteresisNormalization(self, on):
        self._hysteresisNormalize = on is not False

    def setJitterMode(self, mode):
        self._jitterMode = _normalize_jitter_mode(mode)

    def getJitterMode(self):
        return self._jitterMode

    def setRayBudget(self, rays, maxProbesPerTick=None):
        self._rayBudget = int(min(MAX_RAY_BUDGET if maxProbesPerTick is None else 1 << 30, max(2048, int(rays))))
        if maxProbesPerTick is not None:
            self._maxProbesPerTick = max(1, int(maxProbesPerTick))

    def getRayBudget(self):
        return self._rayBudget

    def setRadianceClamp(self, v):
        self._params.radianceClamp = max(0.0, float(v))

    def setDepthSharpness(self, v):
        self._params.depthSharpness = max(0.01, float(v))

    def setFilterStrength(self, v):
        self._params.filterStrength = min(1.0, max(0.0, float(v)))

    def setSmoothness(self, v):
        self._params.filterSmooth = min(1.0, max(0.0, float(v)))

    def setSky(self, sh9=None):
        """setSky (gi_probes.js:1312-1318): nine SH coefficients x RGB; None
        clears the sky and marks it unconfigured (no reflection sky fallback)."""
        sh = np.zeros(27, np.float32) if sh9 is None else np.asarray(sh9, np.float32).reshape(27)
        for i in range(27):
            self._params.skySH[i] = float(sh[i])
        self._params.skyConfigured = 0.0 if sh9 is None else 1.0

    def setReflectionSkyFallback(self, on):
        """A true miss feeds the reflection lobes with the sky (gi_probes.js:1320-1324)."""
        self._params.reflectionSkyFallback = 1.0 if on is True else 0.0

    def getReflectionSkyFallback(self):
        return self._params.reflectionSkyFallback > 0.5

    def getReflectionQuality(self) -> str:
        return self._reflection

    def reflectionLayout(self, ci: int = 0) -> dict:
        """The cascade's reflection layout: tier, glossy tile geometry and the
        glossy phase of its next solve."""
        lay = _abi.sb_reflection_layout()
        self._ck(self._lib.sb_get_reflection_layout(self._ctx, ci, C.byref(lay)))
        return {n: int(getattr(lay, n)) for n, _ in lay._fields_}

    def setSkyIntensity(self, v):
        self._params.skyIntensity = max(0.0, float(v))

    def setNirSensing(self, on):
        self._params.nirGate = 1.0 if on else 0.0

    def setDebugKnobs(self, **knobs):
        for k, v in knobs.items():
            if k == "frameJitter":
                self._frameJitterOverride = None if v is None else float(v)
            elif hasattr(self._params, k):
                setattr(self._params, k, float(v))
            else:
                raise KeyError(k)

    def getResolution(self):
        return tuple(self._res)

    def getRays(self):
        return self._rays

    def getStats(self):
        st = _abi.sb_stats()
        self._ck(self._lib.sb_get_stats(self._ctx, C.byref(st)))
        d = dict(self.stats)
        d.update(probeTotal=self._probeTotal, rays=self._rays, lastSolveMs=st.lastSolveMs,
                 sceneBvhActive=bool(st.sceneBvhActive), sceneBvhBuilding=bool(st.sceneBvhBuilding),
                 sceneBvhBuilds=int(st.sceneBvhBuilds))
        return d

    # ----------------------------------------------------------- scene BVH
    def rebuildSceneBvh(self):
        """Rebuild the scene BVH over the current placements (the reference's
        idle-gated rebuild, gi_probes.js:3269-3455); never needed for correctness."""
        self._ck(self._lib.sb_rebuild_scene_bvh(self._ctx))

    def setSceneBvhBuild(self, mode: str):
        """'blocking': a rebuild completes inside the next tick. 'background': the
        next tick starts it on a host thread and ticks use the two-level walk
        until a later tick installs it."""
        if mode not in SCENE_BVH_BUILD_MODES:
            raise ValueError("sceneBvhBuild: 'blocking' or 'background'")
        self._ck(self._lib.sb_set_scene_bvh_build_mode(self._ctx, SCENE_BVH_BUILD_MODES[mode]))

    def finishSceneBvh(self):
        """Wait for a background scene-BVH build and install it."""
        self._ck(self._lib.sb_finish_scene_bvh(self._ctx))

    # ------------------------------------------------------------- read-back
    def synchronize(self):
        self._ck(self._lib.sb_synchronize(self._ctx))

    def _read_target(self, which: str, out: np.ndarray | None):
        r = self._res
        W, H = r[0] * TILE, r[1] * r[2] * TILE
        P = self._probeTotal
        shapes = {"atlas": ((H, W, 4), np.uint16, "IRRADIANCE_ATLAS"),
                  "depthAtlas": ((H, W, 4), np.uint16, "DEPTH_ATLAS"),
                  "irr": ((P * 64, 4), np.float32, "IRRADIANCE_HISTORY"),
                  "depth": ((P * 64, 2), np.float32, "DEPTH_HISTORY")}
        shape, dt, key = shapes[which]
        if out is None:
            out = np.zeros(shape, dt)
        assert out.shape == shape and out.dtype == dt and out.flags["C_CONTIGUOUS"]
        return key, out

    def _debugRead(self, which: str, cascade: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Read a device buffer (the _debugRead seam, gi_probes.js:4830-4841).
        `out` may be a preallocated (e.g. page-locked) array of the right shape."""
        key, out = self._read_target(which, out)
        self._ck(self._lib.sb_read_buffer(self._ctx, _abi.BUF[key] | (cascade << 8), 0, out.size, _abi.ptr(out)))
        return out

    def _debugReadMany(self, reads, cascade: int = 0) -> list:
        """Several reads queued back to back behind the pending work and waited
        for once: `reads` is a list of (which, out) as for _debugRead."""
        outs = []
        for which, out in reads:
            key, out = self._read_target(which, out)
            self._ck(self._lib.sb_read_buffer_async(self._ctx, _abi.BUF[key] | (cascade << 8), 0, out.size,
                                                    _abi.ptr(out)))
            outs.append(out)
        self.synchronize()
        return outs

    @property
    def ctx(self):
        return self._ctx

    @property
    def pool(self):
        return self._pool

    @property
    def grid(self):
        return self._grid

    def dispose(self):
        if self._disposed:
            return
        self._disposed = True
        self._lib.sb_destroy(self._ctx)
        self._ctx = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


def createProbeField(scene: SceneDesc, **opts) -> ProbeField:
    return ProbeField(scene, **opts)


class SpeedballGIHandle:
    """The object installSpeedballGI returns (install.js:362-503), update path only."""

    def __init__(self, field: ProbeField, onError=None):
        self._gi = field
        self._onError = onError
        self._disposed = False
        self._failureWarned = False
        self.advanced = {"field": field, "tick": field.tick, "setDebugKnobs": field.setDebugKnobs,
                         "debug": {"read": field._debugRead, "state": field.getStats}}

    def update(self, camera=None, playing=False):
        """install.js:364-385: tick, and report failures once per failure streak."""
        if self._disposed:
            return None
        try:
            r = self._gi.tick(playing=playing)
            self._failureWarned = False
            return r
        except Exception as e:  # routed like the reference's promise rejection
            if self._failureWarned:
                return None
            self._failureWarned = True
            if self._onError:
                self._onError(e)
            return None

    def __getattr__(self, name):
        gi = self.__dict__.get("_gi")
        if gi is None or name.startswith("_"):
            raise AttributeError(name)
        target = getattr(gi, name)
        if callable(target) and name.startswith(("set", "mark", "notify")):
            def guarded(*a, **k):
                if self._disposed:
                    return None
                return target(*a, **k)
            return guarded
        return target

    def dispose(self):
        if self._disposed:
            return
        self._disposed = True
        self._gi.dispose()


def installSpeedballGI(scene: SceneDesc, *, enabled=True, intensity=10, divisions=16, rays=64, cascades=2,
                       hysteresis=None, jitterMode="gated", roughReflections=False, reflectionQuality=None,
                       reflectionSkyFallback=False, clusteredLighting=False, volumes=None, device=0,
                       onError=None, **_ignored) -> SpeedballGIHandle:
    """install.js:216-239 with the renderer/camera replaced by the scene description."""
    if onError is not None and not callable(onError):
        raise TypeError("installSpeedballGI: onError must be a function when provided.")
    field = createProbeField(scene, intensity=intensity, hysteresis=hysteresis, jitterMode=jitterMode,
                             divisions=divisions, rays=rays, cascades=cascades, clusteredLighting=clusteredLighting,
                             volumes=volumes, device=device, reflectionQuality=reflectionQuality,
                             roughReflections=roughReflections, reflectionSkyFallback=reflectionSkyFallback)
    return SpeedballGIHandle(field, onError)
