"""Shared set-up for the GPU parity tests: one scene on the CUDA path and the
same scene, grid, lights and parameters on the oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np

from speedball_b200 import _abi
from speedball_b200.field import ProbeField

import orc

# Parity tolerances of the update path: hit t 1e-5 relative, texels
# 1e-3 relative; near-tie exemption when the two nearest candidates are within
# 1e-6 relative.
T_REL = 1e-5
TEXEL_REL = 1e-3
TIE_REL = 1e-6


def grid_dict(g: _abi.sb_grid) -> dict:
    return dict(gridMin=[g.gridMin[a] for a in range(3)], gridSize=[g.gridSize[a] for a in range(3)],
                res=[g.res[a] for a in range(3)], rays=g.raysPerProbe, maxDist=g.maxDist, cellMin=g.cellMin)


def make_field(scene, record=True, rays=None) -> ProbeField:
    m = scene.meta
    g = m["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]),
                   rays=rays or g["rays"], clusteredLighting=m.get("clustered", False),
                   hysteresis=m.get("hysteresis"), jitterMode=m.get("jitter", "gated"), recordHits=record)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)  # one solve covers every probe
    return f


def read(field: ProbeField, key: str, count: int, dtype, cascade: int = 0) -> np.ndarray:
    out = np.zeros(count, dtype)
    _abi.check(field._lib.sb_read_buffer(field.ctx, _abi.BUF[key] | (cascade << 8), 0, count, _abi.ptr(out)),
               field.ctx)
    return out


class OracleMirror:
    """The oracle's copy of a field's scene, grid, lights and FP64 state."""

    def __init__(self, field: ProbeField, fp32: bool = False):
        self.field = field
        pool = field.pool
        self.pool = pool
        self.materials = read(field, "MATERIALS", pool.materials.shape[0], np.float32)
        self.nodes = read(field, "BVH_NODES", pool.bvhNodes.size, np.uint32).reshape(-1, 8)
        self.vertex = read(field, "VERTEX_DATA", pool.vertexData.size, np.float32).reshape(-1, 8)
        self.keep = []
        self.scene = orc.scene_struct(pool, self.materials, nodes=self.nodes, vertex=self.vertex, keep=self.keep)
        self.gdict = grid_dict(field.grid)
        self.grid = orc.grid_struct(self.gdict)
        sc = field._scene
        from speedball_b200.field import selectGiLightRecords
        g = self.gdict
        recs, analytic, _ = selectGiLightRecords(sc.lights, field._clustered, g["gridMin"],
                                                 [g["gridMin"][a] + g["gridSize"][a] for a in range(3)])
        self.light_count = recs.shape[0]
        self.clustered = field._clustered
        self.arena = orc.light_arena(recs, self.clustered, g)
        self.fp32 = fp32
        self.irr, self.depth, self.atlas, self.depth_atlas = orc.new_state(g, fp32)

    def params(self) -> np.ndarray:
        return self.field._params.to_array()

    def solve(self, offset: int, updated: int, replay: dict | None = None, want: bool = True):
        n = updated * self.gdict["rays"]
        io = orc.OrcSolveIO()
        out = {}
        if want:
            out = dict(rays=np.zeros(n * 4, np.float32 if self.fp32 else np.float64), tri=np.zeros(n, np.int32),
                       inst=np.zeros(n, np.int32), second=np.zeros(n, np.float32 if self.fp32 else np.float64),
                       tested=np.zeros(n, np.uint64), blocked=np.zeros(n, np.uint64))
            io.rayOut = orc._p(out["rays"]); io.hitTri = orc._p(out["tri"]); io.hitInst = orc._p(out["inst"])
            io.secondT = orc._p(out["second"]); io.tested = orc._p(out["tested"]); io.blocked = orc._p(out["blocked"])
        if replay is not None:
            io.replayTri = orc._p(replay["tri"]); io.replayInst = orc._p(replay["inst_word"])
            io.replayBlocked = orc._p(replay["blocked"])
        orc.solve(self.scene, self.arena, self.light_count, self.clustered, self.grid, self.grid, self.params(),
                  offset, updated, self.irr, self.depth, self.atlas, self.depth_atlas, fp32=self.fp32, io=io)
        return out


def gpu_records(field: ProbeField, n: int) -> dict:
    hits = read(field, "HIT_RECORDS", n * 4, np.uint32).reshape(n, 4)
    vis = read(field, "VISIBILITY", n * 4, np.uint32).reshape(n, 4)
    tri = hits[:, 0].view(np.int32).copy()
    word = hits[:, 1].copy()
    inst = np.where(tri >= 0, word & 0x7FFFFFFF, 0xFFFFFFFF).astype(np.uint32).view(np.int32)
    t = hits[:, 2].view(np.float32).copy()
    tested = vis[:, 0].astype(np.uint64) | (vis[:, 1].astype(np.uint64) << np.uint64(32))
    unblocked = vis[:, 2].astype(np.uint64) | (vis[:, 3].astype(np.uint64) << np.uint64(32))
    blocked = tested & ~unblocked
    # replay input keeps the facing bit in bit 31 of the instance word
    return dict(tri=np.ascontiguousarray(tri), inst=np.ascontiguousarray(inst),
                inst_word=np.ascontiguousarray(word.view(np.int32)), facing=(word >> 31).astype(bool), t=t,
                blocked=np.ascontiguousarray(blocked))


def half_to_f(a: np.ndarray) -> np.ndarray:
    return a.view(np.float16).astype(np.float64)


def texel_rel_err(g: np.ndarray, o: np.ndarray) -> np.ndarray:
    """|g - o| / max(|o|, floor): relative error with an absolute floor of 1e-3
    of the largest magnitude for near-black texels."""
    floor = max(1e-3 * float(np.abs(o).max()), 1e-12)
    return np.abs(g - o) / np.maximum(np.abs(o), floor)
