"""Scene packing into the reference's pooled layouts.

``build_pool`` is the host half of ``buildSpectralScene`` (spectral_scene.js:1031-2033)
for plain mesh scenes: one local-space BLAS per mesh (built by the library's
host builder, include/speedball_scene.h), pooled into ``bvhNodes``, ``triIndex``,
``vertexData`` (8 floats per vertex) and ``triMaterial`` with pool-absolute miss
links and leaf offsets (1188-1240), the 28-float material records
(materialToUber, 214-307) and room for the instance records + TLAS in the
materials tail (1327-1334). The TLAS itself is built on the GPU
(``sb_build_tlas``) from the instance table returned here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi

MAT_STRIDE = 28
LIGHT_STRIDE = 17
TLAS_STRIDE = 12
MAX_LEAF = 8  # new MeshBVH(..., { targetLeafSize: 8 }), spectral_scene.js:951

# traversal flags, spectral_scene.js:49-51
MAT_FLAG_ALPHA_TEXTURE = 1
MAT_FLAG_ALPHA_ACCEPT = 2
MAT_FLAG_SHADOW_BLOCK = 4


@dataclass
class Mesh:
    positions: np.ndarray            # (V,3) float32, local space
    indices: np.ndarray              # (T,3) uint32
    tri_material: np.ndarray         # (T,) uint32 uber index per triangle
    normals: np.ndarray | None = None
    uvs: np.ndarray | None = None


@dataclass
class Instance:
    mesh: int
    world: np.ndarray                # (4,4) float64, row-major math matrix
    active: bool = True


@dataclass
class SceneDesc:
    meshes: list
    instances: list
    materials: np.ndarray            # (M,28) float32 uber records
    lights: np.ndarray               # (L,17) float32 records
    name: str = "scene"
    meta: dict = field(default_factory=dict)


def material_record(color, roughness=1.0, metalness=0.0, transmission=0.0, ior=1.5, emissive=(0, 0, 0),
                    opacity=1.0, side=0, alpha_test=0.0) -> np.ndarray:
    """materialToUber (spectral_scene.js:214-307) for an untextured material."""
    r, g, b = (float(x) for x in color)
    metal = min(1.0, max(0.0, metalness))
    transm = min(1.0, max(0.0, transmission))
    constant_alpha_ok = opacity > 1.0e-4 and (alpha_test <= 0 or opacity >= alpha_test)
    flags = (MAT_FLAG_ALPHA_ACCEPT if constant_alpha_ok else 0) | (MAT_FLAG_SHADOW_BLOCK if transm < 0.5 else 0)
    rec = [r, g, b, min(1.0, max(0.0, roughness)), metal, transm, max(1.0, ior),
           emissive[0], emissive[1], emissive[2], min(1.0, max(0.0, opacity)), 0.0,
           -1, -1, -1, -1, -1, 1.0, 1.0, 1.0, 0.0, 0.0, float(min(2, max(0, int(side)))),
           min(1.0, max(0.0, alpha_test)), -1, -1, float(flags), 0.0]
    return np.array(rec, dtype=np.float32)


def light_record(kind, pos=(0, 0, 0), direction=(0, 0, -1), color=(1, 1, 1), intensity=1.0, range_=0.0,
                 decay=2.0, cos_angle=-1.0, cos_penumbra=-1.0) -> np.ndarray:
    """One 17-float record of collectLights (spectral_scene.js:724-813).

    kind: 0 directional, 1 point, 2 spot. `direction` points toward the target."""
    c = [color[0] * intensity, color[1] * intensity, color[2] * intensity]
    return np.array([kind, *pos, *direction, *c, range_, decay, cos_angle, cos_penumbra, 0, 0, 0], dtype=np.float32)


def tlas_node_count(n: int) -> int:
    """Nodes of buildTlasRecords' median split with leaf size 2 (spectral_scene.js:973-1003)."""
    t = [1] * (n + 1)
    for m in range(3, n + 1):
        t[m] = 1 + t[m >> 1] + t[m - (m >> 1)]
    return t[n] if n else 0


def build_blas(mesh: Mesh, ctx=None, lib=None):
    """One mesh's BLAS in the threaded layout: on the host (sbh_build_blas), or
    on the GPU of context `ctx` (sb_build_blas_gpu, a linear BVH)."""
    lib = lib or _abi.load()
    pos = np.ascontiguousarray(mesh.positions, dtype=np.float32)
    idx = np.ascontiguousarray(mesh.indices, dtype=np.uint32)
    T = idx.shape[0]
    nodes = np.zeros((2 * T, 8), dtype=np.uint32)
    order = np.zeros(T, dtype=np.uint32)
    if ctx is not None:
        n = C.c_uint32(0)
        _abi.check(lib.sb_build_blas_gpu(ctx, _abi.ptr(pos), pos.shape[0], _abi.ptr(idx), T, MAX_LEAF,
                                         _abi.ptr(nodes), _abi.ptr(order), C.byref(n)), ctx)
        n = n.value
    else:
        n = lib.sbh_build_blas(_abi.ptr(pos), pos.shape[0], _abi.ptr(idx), T, MAX_LEAF, _abi.ptr(nodes),
                               _abi.ptr(order))
    if n == 0:
        raise ValueError("BLAS build failed (empty mesh or out-of-range index)")
    return nodes[:n].copy(), order


@dataclass
class Pool:
    """The typed arrays of buildSpectralScene plus the instance table."""
    bvhNodes: np.ndarray       # (N,8) uint32
    triIndex: np.ndarray       # (T,3) uint32
    vertexData: np.ndarray     # (V,8) float32
    triMaterial: np.ndarray    # (T,) uint32
    materials: np.ndarray      # float32: ubers | instances | TLAS
    materialCount: int
    instBase: int
    instCount: int
    tlasBase: int
    tlasNodeCount: int
    blas_root: np.ndarray      # per mesh
    blas_end: np.ndarray
    vert_base: np.ndarray      # per mesh
    vert_count: np.ndarray
    tri_base: np.ndarray
    tri_count: np.ndarray
    inst_world: np.ndarray     # (I,16) float64, column-major (three Matrix4.elements)
    inst_active: np.ndarray    # (I,) uint8
    inst_root: np.ndarray      # (I,) uint32
    inst_end: np.ndarray

    def view(self) -> _abi.sb_scene_view:
        v = _abi.sb_scene_view()
        v.bvhNodes = _abi.ptr(self.bvhNodes)
        v.nodeCount = self.bvhNodes.shape[0]
        v.triIndex = _abi.ptr(self.triIndex)
        v.triCount = self.triIndex.shape[0]
        v.vertexData = _abi.ptr(self.vertexData)
        v.vertexCount = self.vertexData.shape[0]
        v.triMaterial = _abi.ptr(self.triMaterial)
        v.materials = _abi.ptr(self.materials)
        v.materialsLen = self.materials.shape[0]
        v.materialCount = self.materialCount
        v.instBase = self.instBase
        v.instCount = self.instCount
        v.tlasBase = self.tlasBase
        v.tlasNodeCount = 0  # built on the GPU
        return v


def column_major(m4: np.ndarray) -> np.ndarray:
    """Row-major 4x4 math matrix -> three's column-major elements."""
    return np.ascontiguousarray(np.asarray(m4, dtype=np.float64).T.reshape(16))


def build_pool(scene: SceneDesc, ctx=None, lib=None) -> Pool:
    """The pool of `scene`; with a context, every BLAS is built on its GPU."""
    blas = [build_blas(m, ctx, lib) for m in scene.meshes]
    nV = sum(m.positions.shape[0] for m in scene.meshes)
    nT = sum(m.indices.shape[0] for m in scene.meshes)
    nN = sum(b[0].shape[0] for b in blas)
    if nT >= 1 << 24 or nN >= 1 << 24:
        raise ValueError("BVH pool exceeds the 24-bit index ceiling")
    vertexData = np.zeros((nV, 8), dtype=np.float32)
    triIndex = np.zeros((nT, 3), dtype=np.uint32)
    triMaterial = np.zeros(nT, dtype=np.uint32)
    nodes = np.zeros((nN, 8), dtype=np.uint32)
    M = len(scene.meshes)
    vb = np.zeros(M, np.uint32); vc = np.zeros(M, np.uint32); tb = np.zeros(M, np.uint32); tc = np.zeros(M, np.uint32)
    root = np.zeros(M, np.uint32); end = np.zeros(M, np.uint32)
    v0 = t0 = n0 = 0
    for i, (mesh, (bn, order)) in enumerate(zip(scene.meshes, blas)):
        V, T, N = mesh.positions.shape[0], mesh.indices.shape[0], bn.shape[0]
        vertexData[v0:v0 + V, 0:3] = mesh.positions
        if mesh.normals is not None:
            vertexData[v0:v0 + V, 3:6] = mesh.normals
        if mesh.uvs is not None:
            vertexData[v0:v0 + V, 6:8] = mesh.uvs
        triIndex[t0:t0 + T] = mesh.indices[order] + v0
        triMaterial[t0:t0 + T] = mesh.tri_material[order]
        b = bn.copy()
        b[:, 6] += n0
        leaf = b[:, 7] != 0xFFFFFFFF
        b[leaf, 7] = (b[leaf, 7] & 0xFF000000) | ((b[leaf, 7] & 0x00FFFFFF) + t0)
        nodes[n0:n0 + N] = b
        vb[i], vc[i], tb[i], tc[i], root[i], end[i] = v0, V, t0, T, n0, n0 + N
        v0 += V; t0 += T; n0 += N
    ubers = np.asarray(scene.materials, dtype=np.float32).reshape(-1, MAT_STRIDE)
    I = len(scene.instances)
    tlasN = tlas_node_count(I)
    instBase = ubers.shape[0] * MAT_STRIDE
    tlasBase = instBase + I * MAT_STRIDE
    materials = np.zeros(tlasBase + tlasN * TLAS_STRIDE, dtype=np.float32)
    materials[:instBase] = ubers.reshape(-1)
    world = np.zeros((I, 16), np.float64)
    active = np.zeros(I, np.uint8)
    iroot = np.zeros(I, np.uint32); iend = np.zeros(I, np.uint32)
    for k, inst in enumerate(scene.instances):
        world[k] = column_major(inst.world)
        active[k] = 1 if inst.active else 0
        iroot[k] = root[inst.mesh]
        iend[k] = end[inst.mesh]
    return Pool(nodes, triIndex, vertexData, triMaterial, materials, ubers.shape[0], instBase, I, tlasBase, tlasN,
                root, end, vb, vc, tb, tc, world, active, iroot, iend)
