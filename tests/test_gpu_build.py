"""GPU BLAS build (sb_build_blas_gpu / sb_build_blas_device): a linear BVH
emitted in the reference's threaded layout, checked against the oracle.

Per mesh: the oracle's refitFlatBlasRange restatement accepts the layout (the
threaded-layout contract of gi_refit.js:96-139) and leaves every node's
bounds bit-identical (a build's bounds are the exact min/max a refit gives);
leaves hold 1..8 triangles and cover every BVH position exactly once; the
triangle order is a permutation. Meshes: the room's icospheres, atrium meshes
of 500 to 60k triangles, and edge cases (one triangle, two, nine, every
centroid equal). Scene level: a field whose BLASes are all GPU-built gives the
FP64 oracle's closest hits (every difference explained ray by ray) and replays
a solve within 1e-3 per texel.
"""
import ctypes as C
import time

import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth
from speedball_b200.scene import Mesh

import gpu_util as gu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.sb_create(C.byref(_abi.sb_device_opts(0, 0)), C.byref(h)))
    yield lib, h
    lib.sb_destroy(h)


def _gpu_build(lib, h, mesh, leaf=8):
    pos = np.ascontiguousarray(mesh.positions, np.float32)
    idx = np.ascontiguousarray(mesh.indices, np.uint32)
    T = idx.shape[0]
    nodes = np.zeros((2 * T, 8), np.uint32)
    order = np.zeros(T, np.uint32)
    n = C.c_uint32(0)
    _abi.check(lib.sb_build_blas_gpu(h, _abi.ptr(pos), pos.shape[0], _abi.ptr(idx), T, leaf, _abi.ptr(nodes),
                                     _abi.ptr(order), C.byref(n)), h)
    return nodes[:n.value].copy(), order


def _check_layout(mesh, nodes, order, leaf=8):
    T = mesh.indices.shape[0]
    n = nodes.shape[0]
    assert 1 <= n <= 2 * T - 1
    assert np.array_equal(np.sort(order), np.arange(T, dtype=np.uint32))
    lf = nodes[:, 7] != 0xFFFFFFFF
    cnt = nodes[lf, 7] >> 24
    off = nodes[lf, 7] & 0xFFFFFF
    assert cnt.min() >= 1 and cnt.max() <= leaf
    covered = np.concatenate([np.arange(o, o + c) for o, c in zip(off, cnt)])
    assert np.array_equal(np.sort(covered), np.arange(T))
    assert np.all(nodes[:, 6] > np.arange(n)) and np.all(nodes[:, 6] <= n)
    # the oracle's refit accepts the layout and reproduces every bound bit for bit
    tri = np.ascontiguousarray(mesh.indices[order], np.uint32)
    vd = np.zeros((mesh.positions.shape[0], 8), np.float32)
    vd[:, 0:3] = mesh.positions
    re = nodes.copy()
    assert orc.load().orc_refit_blas(orc._p(re), re.size, orc._p(tri), tri.size, orc._p(vd), vd.size, 0, n) == 1
    assert np.array_equal(re, nodes)


def _edge_meshes():
    rng = np.random.default_rng(3)
    out = []
    for T in (1, 2, 9):
        P = rng.uniform(-1, 1, (3 * T, 3)).astype(np.float32)
        out.append(Mesh(P, np.arange(3 * T, dtype=np.uint32).reshape(T, 3), np.zeros(T, np.uint32)))
    # 40 triangles sharing one bounds centre (equal Morton codes throughout)
    base = rng.uniform(-1, 1, (3, 3)).astype(np.float32)
    P = np.concatenate([base * s for s in np.linspace(0.5, 2.0, 40, dtype=np.float32)])
    out.append(Mesh(P.astype(np.float32), np.arange(120, dtype=np.uint32).reshape(40, 3), np.zeros(40, np.uint32)))
    return out


def test_gpu_blas_layout_and_bounds(ctx):
    lib, h = ctx
    meshes = synth.room_spheres(0).meshes[:8] + synth.atrium(1).meshes[:12] + _edge_meshes()
    sizes = []
    for m in meshes:
        nodes, order = _gpu_build(lib, h, m)
        _check_layout(m, nodes, order)
        sizes.append((m.indices.shape[0], nodes.shape[0]))
    print("triangles -> nodes:", sizes)


def test_gpu_blas_build_time(ctx):
    """The largest archetype of the large scene (600k triangles): GPU build
    against the host builder (reported; the reference's CPU MeshBVH build of a
    large mesh is ~200 ms, spectral_scene.js / CHANGELOG)."""
    lib, h = ctx
    from speedball_b200 import scene as sc
    s = synth.large_scene()
    m = max(s.meshes, key=lambda x: x.indices.shape[0])
    _gpu_build(lib, h, m)  # warm-up: scratch allocation
    t0 = time.perf_counter()
    nodes, order = _gpu_build(lib, h, m)
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    sc.build_blas(m)
    t_host = time.perf_counter() - t0
    print(f"{m.indices.shape[0]} triangles: GPU build {t_gpu * 1e3:.1f} ms (host arrays in/out), "
          f"host build {t_host * 1e3:.1f} ms, {nodes.shape[0]} nodes")
    _check_layout(m, nodes, order)


def test_scene_with_gpu_built_blases_matches_oracle():
    from speedball_b200.field import ProbeField
    s = synth.room_spheres(0)
    g = s.meta["grid"]
    f = ProbeField(s, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1, rays=g["rays"],
                   hysteresis=s.meta.get("hysteresis"), recordHits=True, blasBuilder="gpu")
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
    try:
        mirror = gu.OracleMirror(f)
        rng = np.random.default_rng(17)
        n = 100_000
        ro = rng.uniform(0.3, 9.7, (n, 3)).astype(np.float32)
        rd = rng.normal(size=(n, 3))
        rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
        t = np.zeros(n, np.float32); tri = np.zeros(n, np.int32); inst = np.zeros(n, np.int32)
        _abi.check(f._lib.sb_raycast(f.ctx, _abi.ptr(ro), _abi.ptr(rd), n, _abi.ptr(t), _abi.ptr(tri), _abi.ptr(inst)),
                   f.ctx)
        ot, otri, oinst, o2 = np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        orc.load().orc_closest(C.byref(mirror.scene), orc._p(ro), orc._p(rd), n, 1, 0, orc._p(ot), orc._p(otri),
                               orc._p(oinst), orc._p(o2), orc.threads())
        gu.check_hits(mirror.scene, ro.astype(np.float64), rd.astype(np.float64), tri, inst, t, otri, oinst, ot)
        frame = f.tick()
        f.synchronize()
        gu.solve_parity(f, mirror, frame, f._params.to_array())
    finally:
        f.dispose()
