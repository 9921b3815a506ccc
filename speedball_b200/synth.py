"""Seeded synthetic scenes for the probe-update workloads.

No public dataset is involved: the reference's Sponza mesh is absent from its
tree, so the 262k-triangle atrium below stands in for it at the same scale.
Every scene is a pure function of its seed (numpy PCG64).

  room_spheres   10 m box room (12 triangles) + 64 icospheres (subdivision 3,
                 1280 triangles, radius U[0.2,0.8]); one BLAS per mesh, 65
                 instances; 16 Lambertian materials; 1 directional + 4 point
                 lights; 8^3 probes, 64 rays.
  atrium         262,267 triangles in 30 meshes (log-uniform 500-60k) of
                 column prisms, arched wall panels and subdivided floor slabs;
                 25 materials; 1 directional + 32 point lights (clustered);
                 16^3 probes, 64 rays; 3 rigid movers and 1 deforming mesh.
"""
from __future__ import annotations

import math

import numpy as np

from .scene import Instance, Mesh, SceneDesc, light_record, material_record


# ----------------------------------------------------------------- meshes
def icosphere(subdiv: int, radius: float = 1.0):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    P = np.array(verts) * radius
    F = np.array(faces, dtype=np.uint32)
    return P.astype(np.float32), F, (np.array(verts)).astype(np.float32)


def box_room(size: float):
    """Inward-facing box [0,size]^3 (front faces toward the interior)."""
    s = size
    P = np.array([(0, 0, 0), (s, 0, 0), (s, s, 0), (0, s, 0), (0, 0, s), (s, 0, s), (s, s, s), (0, s, s)],
                 dtype=np.float32)
    # outward CCW quads, then reversed for an inward front face
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    F = []
    for a, b, c, d in quads:
        F += [(a, c, b), (a, d, c)]
    return P, np.array(F, dtype=np.uint32)


def grid_mesh(nu: int, nv: int, fn):
    """Parametric grid (nu x nv quads) -> positions and CCW triangles; fn(u, v) -> (x, y, z)."""
    u = np.linspace(0.0, 1.0, nu + 1)
    v = np.linspace(0.0, 1.0, nv + 1)
    U, V = np.meshgrid(u, v, indexing="xy")
    P = np.stack(fn(U, V), axis=-1).reshape(-1, 3).astype(np.float32)
    i = np.arange(nu)[None, :] + (nu + 1) * np.arange(nv)[:, None]
    a, b, c, d = i, i + 1, i + nu + 2, i + nu + 1
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)], 0)
    # interleave so truncation removes whole rows last
    F = np.stack([np.stack([a, b, c], -1), np.stack([a, c, d], -1)], -2).reshape(-1, 3)
    return P, F.astype(np.uint32)


def _dims_for(n_tris: int, aspect: float):
    quads = (n_tris + 1) // 2
    nv = max(1, int(round(math.sqrt(quads / aspect))))
    nu = max(1, -(-quads // nv))
    return nu, nv


def column_prism(n_tris: int, rng):
    """Extruded n-gon column with sinusoidal fluting: a closed tube grid."""
    sides = int(rng.integers(6, 17))
    radius = float(rng.uniform(0.25, 0.7))
    height = float(rng.uniform(4.0, 12.0))
    nu, nv = _dims_for(n_tris, aspect=sides / 4.0)
    flute = float(rng.uniform(0.0, 0.06))

    def fn(u, v):
        a = u * 2 * math.pi
        r = radius * (1.0 + flute * np.cos(a * sides))
        return r * np.cos(a), v * height, r * np.sin(a)
    P, F = grid_mesh(nu, nv, fn)
    return P, F[:n_tris]


def arched_panel(n_tris: int, rng, w=None, h=None):
    """Wall panel with an arched top edge, slightly curved in depth."""
    w = float(rng.uniform(4.0, 12.0)) if w is None else float(w)
    h = float(rng.uniform(4.0, 10.0)) if h is None else float(h)
    arch = float(rng.uniform(0.5, 2.5))
    bow = float(rng.uniform(0.0, 0.6))
    nu, nv = _dims_for(n_tris, aspect=w / h)

    def fn(u, v):
        x = (u - 0.5) * w
        top = h + arch * np.sin(np.pi * u)
        return x, v * top, bow * np.sin(np.pi * u) * (1.0 - v)
    P, F = grid_mesh(nu, nv, fn)
    return P, F[:n_tris]


def floor_slab(n_tris: int, rng, w=None, d=None):
    """Rectangular slab, 2-level subdivided grid with a shallow relief."""
    w = float(rng.uniform(6.0, 20.0)) if w is None else float(w)
    d = float(rng.uniform(6.0, 20.0)) if d is None else float(d)
    relief = float(rng.uniform(0.0, 0.05))
    nu, nv = _dims_for(n_tris, aspect=w / d)

    def fn(u, v):
        return (u - 0.5) * w, relief * np.sin(13.0 * u) * np.cos(11.0 * v), (v - 0.5) * d
    P, F = grid_mesh(nu, nv, fn)
    # slabs face up: CCW seen from +y
    F = F[:, [0, 2, 1]]
    return P, F[:n_tris]


def _rot(axis, ang):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = math.cos(ang), math.sin(ang)
    C = 1 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def trs(t, r=None, s=1.0):
    m = np.eye(4)
    m[:3, :3] = (r if r is not None else np.eye(3)) * s
    m[:3, 3] = t
    return m


# ----------------------------------------------------------------- scenes
def room_spheres(seed: int = 0, n_materials: int = 16, n_point: int = 4, n_dir: int = 1):
    """The 82k-triangle room + 64 icospheres scene (plain DDGI, CPU-checkable size).

    The differentiated workload uses n_materials=64, n_point=32, n_dir=0: 416
    parameters (64 x 3 albedo, 64 x 3 emissive, 32 light intensities)."""
    rng = np.random.default_rng(seed)
    S = 10.0
    meshes, instances = [], []
    mats = [material_record(rng.uniform(0.1, 0.9, 3)) for _ in range(n_materials)]
    P, F = box_room(S)
    meshes.append(Mesh(P, F, np.full(F.shape[0], rng.integers(n_materials), np.uint32)))
    instances.append(Instance(0, np.eye(4)))
    unit, uf, un = icosphere(3)
    for i in range(64):
        r = float(rng.uniform(0.2, 0.8))
        c = rng.uniform(0.0, S, 3)
        m = int(rng.integers(n_materials))
        meshes.append(Mesh(unit * r, uf, np.full(uf.shape[0], m, np.uint32), normals=un))
        instances.append(Instance(len(meshes) - 1, trs(c)))
    lights = []
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    if n_dir:
        lights.append(light_record(0, pos=(5, 5, 5), direction=tuple(d), intensity=3.0))
    for _ in range(n_point):
        lights.append(light_record(1, pos=tuple(rng.uniform(0.0, S, 3)), intensity=float(rng.uniform(5, 20)),
                                   range_=8.0, decay=2.0))
    grid = dict(gridMin=(0.5, 0.5, 0.5), gridSize=(9.0, 9.0, 9.0), res=(8, 8, 8), rays=64)
    return SceneDesc(meshes, instances, np.stack(mats), np.stack(lights), name="room_spheres",
                     meta=dict(grid=grid, clustered=False, hysteresis=0.97, jitter="gated", seed=seed))


def emitter_record(center, radiance, radius: float, proj_area: float) -> np.ndarray:
    """A giEmitter light record (collectEmitterRecords, spectral_scene.js:815-888):
    type 3, centre, surface radiance, range from power, radius, A/4."""
    rng_ = float(np.sqrt(max(0.0, *radiance) * proj_area / 0.005))
    return np.array([3, *center, 0, 0, -1, *radiance, rng_, 2, -1, -1, radius, proj_area, 0], dtype=np.float32)


def add_emitters(scene: SceneDesc, seed: int = 5, sphere: int = 1, points: int = 2) -> SceneDesc:
    """Emissive giEmitter lights for a room scene: icosphere instance `sphere`
    gets its own emissive material and a sphere emitter record (its bounding
    radius and A/4 of its world surface), plus `points` free point-like
    emitters of radius 0 (their visibility rays end at their centres)."""
    rng = np.random.default_rng(seed)
    mats = np.asarray(scene.materials, np.float32).reshape(-1, 28)
    inst = scene.instances[sphere]
    mesh = scene.meshes[inst.mesh]
    radiance = tuple(float(x) for x in rng.uniform(2.0, 6.0, 3))
    rec = material_record((0.8, 0.8, 0.8), emissive=radiance)
    mats = np.concatenate([mats, rec[None]], 0)
    mesh.tri_material = np.full(mesh.indices.shape[0], mats.shape[0] - 1, np.uint32)
    W = np.asarray(inst.world, np.float64)
    P = mesh.positions.astype(np.float64) @ W[:3, :3].T + W[:3, 3]
    tri = P[mesh.indices.astype(np.int64)]
    area = float(np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1).sum() * 0.5)
    center = W[:3, 3]
    radius = float(np.linalg.norm(P - center, axis=1).max())
    recs = [emitter_record(tuple(center), radiance, radius, area / 4.0)]
    for _ in range(points):
        recs.append(emitter_record(tuple(rng.uniform(1.0, 9.0, 3)), tuple(float(x) for x in rng.uniform(2, 5, 3)),
                                   0.0, float(rng.uniform(0.1, 0.4))))
    scene.materials = mats
    scene.lights = np.concatenate([np.asarray(scene.lights, np.float32).reshape(-1, 17), np.stack(recs)], 0)
    scene.meta = dict(scene.meta, emitters=len(recs))
    return scene


ATRIUM_TRIS = 262_267


def atrium(seed: int = 1, total_tris: int = ATRIUM_TRIS, n_meshes: int = 30, n_materials: int = 25,
           n_point: int = 32):
    """Sponza-scale procedural atrium (262,267 triangles in 30 meshes)."""
    rng = np.random.default_rng(seed)
    W, H, D = 40.0, 20.0, 30.0
    raw = np.exp(rng.uniform(math.log(500), math.log(60_000), n_meshes))
    counts = np.maximum(500, np.round(raw * total_tris / raw.sum())).astype(np.int64)
    counts = np.minimum(counts, 60_000)
    diff = total_tris - int(counts.sum())
    order = np.argsort(-counts)
    k = 0
    while diff != 0:
        i = order[k % n_meshes]
        step = max(-diff, min(diff, 60_000 - counts[i])) if diff > 0 else max(diff, 500 - counts[i])
        counts[i] += step
        diff -= step
        k += 1
        if k > 10_000:
            break
    assert counts.sum() == total_tris
    # double-sided (side 2) like most of Sponza's materials in three.js scenes
    mats = [material_record(rng.uniform(0.05, 0.95, 3), side=2) for _ in range(n_materials)]
    meshes, instances = [], []
    kinds = []
    # the five largest meshes close the atrium: a floor slab and four arched
    # perimeter walls facing inward (open to the sky above, like Sponza's court)
    big = [int(i) for i in np.argsort(-counts, kind="stable")[:5]]
    envelope = {big[0]: "floor", big[1]: "wall0", big[2]: "wall1", big[3]: "wall2", big[4]: "wall3"}
    interior = 0
    for i, n in enumerate(counts):
        if i in envelope:
            kind = envelope[i]
        else:
            kind = ["slab", "panel", "column", "column"][interior % 4]
            interior += 1
        if kind == "floor":
            P, F = floor_slab(int(n), rng, w=W, d=D)
            t, R = (W / 2, 0.0, D / 2), _rot((0, 1, 0), 0.0)
        elif kind.startswith("wall"):
            side = int(kind[-1])
            span = W if side < 2 else D
            P, F = arched_panel(int(n), rng, w=span, h=H * 0.8)
            if side == 0:
                t, R = (W / 2, 0.0, 0.0), _rot((0, 1, 0), 0.0)
            elif side == 1:
                t, R = (W / 2, 0.0, D), _rot((0, 1, 0), math.pi)
            elif side == 2:
                t, R = (0.0, 0.0, D / 2), _rot((0, 1, 0), math.pi / 2)
            else:
                t, R = (W, 0.0, D / 2), _rot((0, 1, 0), -math.pi / 2)
        elif kind == "column":
            P, F = column_prism(int(n), rng)
            t = (rng.uniform(2, W - 2), 0.0, rng.uniform(2, D - 2))
            R = _rot((0, 1, 0), rng.uniform(0, 2 * math.pi))
        elif kind == "panel":
            P, F = arched_panel(int(n), rng)
            side = int(rng.integers(4))
            if side == 0:
                t, R = (rng.uniform(6, W - 6), 0.0, 0.3), _rot((0, 1, 0), 0.0)
            elif side == 1:
                t, R = (rng.uniform(6, W - 6), 0.0, D - 0.3), _rot((0, 1, 0), math.pi)
            elif side == 2:
                t, R = (0.3, 0.0, rng.uniform(6, D - 6)), _rot((0, 1, 0), math.pi / 2)
            else:
                t, R = (W - 0.3, 0.0, rng.uniform(6, D - 6)), _rot((0, 1, 0), -math.pi / 2)
        else:
            P, F = floor_slab(int(n), rng)
            level = float(rng.choice([0.05, 6.0, 12.0]))
            t = (rng.uniform(8, W - 8), level, rng.uniform(8, D - 8))
            R = _rot((0, 1, 0), rng.uniform(0, 2 * math.pi))
        assert F.shape[0] == n, (kind, F.shape[0], n)
        m = int(rng.integers(n_materials))
        meshes.append(Mesh(P, F, np.full(F.shape[0], m, np.uint32)))
        instances.append(Instance(i, trs(t, R)))
        kinds.append(kind)
    lights = []
    d = np.array([0.3, -1.0, 0.2])
    d /= np.linalg.norm(d)
    lights.append(light_record(0, pos=(W / 2, H, D / 2), direction=tuple(d), intensity=2.0))
    for _ in range(n_point):
        lights.append(light_record(1, pos=(rng.uniform(1, W - 1), rng.uniform(0.5, H - 0.5), rng.uniform(1, D - 1)),
                                   intensity=float(rng.uniform(20, 120)), range_=float(rng.uniform(5, 12)),
                                   decay=2.0))
    movers = [int(i) for i in rng.choice([i for i, k in enumerate(kinds) if k == "column"], 3, replace=False)]
    candidates = [i for i in range(n_meshes) if i not in movers and i not in envelope]
    deformer = min(candidates, key=lambda i: abs(int(counts[i]) - 20_000))
    grid = dict(gridMin=(0.5, 0.25, 0.5), gridSize=(W - 1.0, H - 0.5, D - 1.0), res=(16, 16, 16), rays=64)
    return SceneDesc(meshes, instances, np.stack(mats), np.stack(lights), name="atrium",
                     meta=dict(grid=grid, clustered=True, hysteresis=0.97, jitter="gated", seed=seed,
                               movers=movers, deformer=deformer, kinds=kinds))


def atrium_motion(scene: SceneDesc, frame: int, seed: int = 7):
    """Per-frame motion: new world matrices for the 3 movers and the deformed
    positions of the deforming mesh (sinusoidal offset, amplitude 2 cm)."""
    rng = np.random.default_rng(seed * 1_000_003 + frame)
    mats = {}
    for i in scene.meta["movers"]:
        base = scene.instances[i].world
        ang = rng.uniform(-0.2, 0.2)
        off = rng.uniform(-0.5, 0.5, 3) * np.array([1.0, 0.0, 1.0])
        m = base.copy()
        m[:3, :3] = _rot((0, 1, 0), ang) @ base[:3, :3]
        m[:3, 3] = base[:3, 3] + off
        mats[i] = m
    dm = scene.meshes[scene.meta["deformer"]]
    P = dm.positions.astype(np.float64)
    ph = 0.35 * frame
    offs = 0.02 * np.sin(P[:, 0] * 1.7 + ph) * np.cos(P[:, 2] * 1.3 + 0.5 * ph)
    Pn = P.copy()
    Pn[:, 1] += offs
    return mats, Pn.astype(np.float32)


LARGE_ARCHETYPE_TRIS = (2_000, 9_000, 40_000, 120_000, 230_000, 500_000, 600_000, 600_000)
LARGE_INSTANCES = (220, 110, 45, 1, 12, 5, 4, 3)   # 400 instances; archetype 3 is the skinned mesh
LARGE_BONES = 8


def skinned_tube(n_tris: int, rng, bones: int = LARGE_BONES, height: float = 12.0, radius: float = 1.2):
    """A closed tube along +y with a chain of `bones` joints at even heights:
    per vertex the two nearest joints and a linear weight between them."""
    sides = 24
    nu, nv = _dims_for(n_tris, aspect=sides / 8.0)

    def fn(u, v):
        a = u * 2 * math.pi
        r = radius * (1.0 + 0.08 * np.cos(a * 5) + 0.15 * np.sin(v * 9.0))
        return r * np.cos(a), v * height, r * np.sin(a)
    P, F = grid_mesh(nu, nv, fn)
    F = F[:n_tris]
    seg = height / bones
    s = np.clip(P[:, 1] / seg - 0.5, 0.0, bones - 1.0)
    b0 = np.floor(s).astype(np.int32)
    b1 = np.minimum(b0 + 1, bones - 1)
    w1 = (s - b0).astype(np.float32)
    joints = np.array([[0.0, seg * (j + 0.5), 0.0] for j in range(bones)], np.float64)
    return P, F, dict(b0=b0, b1=b1, w1=w1, joints=joints)


def skin(rest: np.ndarray, rig: dict, angles: np.ndarray) -> np.ndarray:
    """Linear blend skinning of the tube: joint j rotates its subchain by
    angles[j] (axis-angle vectors, radians) about the joint; each vertex blends
    the world transforms of its two joints."""
    J = rig["joints"]
    n = J.shape[0]
    Rw = [np.eye(3)]
    tw = [np.zeros(3)]
    R_acc, t_acc = np.eye(3), np.zeros(3)
    mats = []
    for j in range(n):
        ang = float(np.linalg.norm(angles[j]))
        Rj = _rot(angles[j] / ang, ang) if ang > 0 else np.eye(3)
        # rotation about joint j applied after the parent chain
        pj = R_acc @ J[j] + t_acc
        R_acc = Rj @ R_acc
        t_acc = Rj @ (t_acc - pj) + pj
        mats.append((R_acc.copy(), t_acc.copy()))
    P = rest.astype(np.float64)
    out = np.empty_like(P)
    w1 = rig["w1"].astype(np.float64)[:, None]
    for j in range(n):
        R, t = mats[j]
        Q = P @ R.T + t
        m0 = rig["b0"] == j
        m1 = rig["b1"] == j
        out[m0] = Q[m0] * (1.0 - w1[m0])
        # second joint's share added below
    for j in range(n):
        R, t = mats[j]
        m1 = rig["b1"] == j
        out[m1] += (P[m1] @ R.T + t) * w1[m1]
    return out.astype(np.float32)


def large_scene(seed: int = 4):
    """The large workload: 8 archetypes of 2k-600k triangles (2.1M unique),
    400 instances scattered over a 160 x 40 x 160 m world, archetype 3 a
    120k-triangle skinned tube (one instance) refit every frame, 64 point
    lights (clustered), 32^3 probes x 256 rays."""
    rng = np.random.default_rng(seed)
    W, Hh, D = 160.0, 40.0, 160.0
    n_materials = 32
    mats = [material_record(rng.uniform(0.05, 0.95, 3), side=2) for _ in range(n_materials)]
    meshes, instances = [], []
    rig = None
    for a, n in enumerate(LARGE_ARCHETYPE_TRIS):
        if a == 3:
            P, F, rig = skinned_tube(int(n), rng)
        elif a in (6, 7):
            P, F = floor_slab(int(n), rng, w=W if a == 6 else 40.0, d=D if a == 6 else 40.0)
        elif a == 5:
            P, F = arched_panel(int(n), rng, w=30.0, h=20.0)
        elif a in (2, 4):
            P, F = column_prism(int(n), rng)
        else:
            P, F = arched_panel(int(n), rng) if a == 1 else column_prism(int(n), rng)
        assert F.shape[0] == n, (a, F.shape[0], n)
        meshes.append(Mesh(P, F, np.full(F.shape[0], int(rng.integers(n_materials)), np.uint32)))
    skinned_instance = -1
    for a, count in enumerate(LARGE_INSTANCES):
        for k in range(count):
            if a == 6 and k == 0:
                m = trs((W / 2, 0.0, D / 2))  # the ground
            else:
                s = float(rng.uniform(0.6, 1.6)) if a not in (6, 7) else 1.0
                t = (rng.uniform(4, W - 4), rng.uniform(0.0, 2.0) if a in (6, 7) else 0.0, rng.uniform(4, D - 4))
                m = trs(t, _rot((0, 1, 0), rng.uniform(0, 2 * math.pi)), s)
            if a == 3:
                skinned_instance = len(instances)
            instances.append(Instance(a, m))
    lights = []
    for _ in range(64):
        lights.append(light_record(1, pos=(rng.uniform(2, W - 2), rng.uniform(1.0, Hh - 2), rng.uniform(2, D - 2)),
                                   intensity=float(rng.uniform(40, 200)), range_=float(rng.uniform(10, 24)),
                                   decay=2.0))
    grid = dict(gridMin=(2.0, 0.5, 2.0), gridSize=(W - 4.0, Hh - 1.0, D - 4.0), res=(32, 32, 32), rays=256)
    return SceneDesc(meshes, instances, np.stack(mats), np.stack(lights), name="large",
                     meta=dict(grid=grid, clustered=True, hysteresis=0.97, jitter="gated", seed=seed,
                               skinned=3, skinnedInstance=skinned_instance, rig=rig))


def large_pose(scene: SceneDesc, frame: int, seed: int = 11, max_deg: float = 15.0) -> np.ndarray:
    """Skinned positions of the large scene's tube for `frame`: every joint
    rotated by a random axis and an angle of at most `max_deg` degrees."""
    rng = np.random.default_rng(seed * 1_000_003 + frame)
    rig = scene.meta["rig"]
    n = rig["joints"].shape[0]
    axes = rng.normal(size=(n, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    ang = np.radians(rng.uniform(0.0, max_deg, n))
    rest = scene.meta.setdefault("restPositions", scene.meshes[scene.meta["skinned"]].positions.copy())
    return skin(rest, rig, axes * ang[:, None])


def large_field(scene: SceneDesc, device: int = 0, recordHits: bool = False):
    """The large scene's probe field: C0 = 32^3 probes x 256 rays over the
    world box; C1 = the fine cascade that fitFineBox places inside it
    (gi_probes.js:3370-3410) at up to 32 probes per axis (divisions 32, so
    the C1 density target 2 x 32 meets the per-axis cap). Clustered lights,
    gated jitter, normalisation off, full updates. A pool whose centroid
    histogram gives no fine box gets the half-extent box around C0's centre."""
    from .field import ProbeField
    g = scene.meta["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=2,
                   divisions=32, rays=g["rays"], clusteredLighting=True, hysteresis=scene.meta["hysteresis"],
                   jitterMode="gated", recordHits=recordHits, device=device)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 30, maxProbesPerTick=1 << 20)
    if not f.hasFineCascade():
        c1 = nested_cascades(g, res=(g["res"], g["res"]), scale=0.5)[1]
        f.configureCascade(1, c1["gridMin"], c1["gridSize"], c1["res"])
    return f


BATCH_SCENE_TRIS = (20_000, 45_000, 80_000, 120_000, 200_000, 262_000, 350_000, 500_000)


def batch_scenes(seed: int = 2, sizes=BATCH_SCENE_TRIS):
    """The batched workload's independent scenes: atria built like the 262k one
    with uneven triangle counts, each with its own cubic probe grid of 8^3 to
    16^3 probes at 32 to 128 rays per probe (multiples of 16) drawn from the
    seed, montecarlo jitter."""
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        s = atrium(seed=100 + i, total_tris=int(n))
        r = int(rng.integers(8, 17))
        rays = int(rng.choice(np.arange(32, 129, 16)))
        s.meta["grid"] = dict(s.meta["grid"], res=(r, r, r), rays=rays)
        s.meta["jitter"] = "montecarlo"
        s.name = f"atrium_{n}"
        out.append(s)
    return out


def nested_cascades(grid: dict, res=((16, 16, 16), (12, 12, 12), (8, 8, 8)), scale: float = 2.0):
    """Cascade boxes sharing a centre, each `scale` times the previous extent."""
    c = np.asarray(grid["gridMin"], np.float64) + 0.5 * np.asarray(grid["gridSize"], np.float64)
    size = np.asarray(grid["gridSize"], np.float64)
    out = []
    for i, r in enumerate(res):
        s = size * scale ** i
        out.append(dict(gridMin=tuple(c - 0.5 * s), gridSize=tuple(s), res=tuple(r), rays=grid["rays"]))
    return out
