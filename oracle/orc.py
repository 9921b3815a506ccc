"""ctypes wrapper of the oracle (liborc.so).

TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference's DDGI
probe-update path that the CUDA library is checked against, and the FP32 CPU
baseline bench.py times. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs may import it. Parity against the reference itself is
unpinned (see orc_core.hpp).
"""
from __future__ import annotations

import ctypes as C
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
    _fields_ = [("data", C.c_void_p), ("dataLen", C.c_uint32), ("lightCount", C.c_uint32), ("clustered", C.c_int32)]


class OrcGrid(C.Structure):
    _fields_ = [("gridMin", C.c_double * 3), ("gridSize", C.c_double * 3), ("res", C.c_uint32 * 3),
                ("rays", C.c_uint32), ("maxDist", C.c_double), ("cellMin", C.c_double)]


class OrcSolveIO(C.Structure):
    _fields_ = [("rayOut", C.c_void_p), ("hitTri", C.c_void_p), ("hitInst", C.c_void_p), ("secondT", C.c_void_p),
                ("tested", C.c_void_p), ("blocked", C.c_void_p), ("replayTri", C.c_void_p),
                ("replayInst", C.c_void_p), ("replayBlocked", C.c_void_p), ("rayIn", C.c_void_p),
                ("preRound", C.c_void_p), ("counters", C.c_void_p), ("hitFacing", C.c_void_p)]


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
          nthreads: int | None = None) -> None:
    lib = load()
    L = OrcLights()
    L.data = _p(arena); L.dataLen = arena.shape[0]; L.lightCount = light_count; L.clustered = 1 if clustered else 0
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
