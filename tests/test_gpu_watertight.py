"""The watertight ray/triangle test (Woop, Benthin & Wald 2013) built as
libspeedball_cuda_watertight.so, beside the reference's Möller–Trumbore test
of the default library.

  * rays aimed exactly at the shared vertices of closed icospheres: with the
    watertight test none passes through the surface; the count for
    Möller–Trumbore is reported beside it;
  * hit IDs against the FP64 oracle (which runs the reference's
    Möller–Trumbore): every difference explained ray by ray (near-tie or an
    edge graze within the FP32 bound), on random rays in the room (config 0)
    and on every probe ray of an atrium solve (config 1); the texels of that
    solve replay on the oracle within 1e-3.
"""
import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu


def _field(scene, variant):
    from speedball_b200.field import ProbeField
    m = scene.meta
    g = m["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1,
                   rays=g["rays"], clusteredLighting=m.get("clustered", False), hysteresis=m.get("hysteresis"),
                   jitterMode="gated", recordHits=True, variant=variant)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
    return f


def test_libraries_report_their_triangle_test():
    assert _abi.load().sb_triangle_test() == 0
    assert _abi.load("watertight").sb_triangle_test() == 1


def _vertex_rays(scene, offset=0.05):
    ro, rd = [], []
    for inst in scene.instances:
        P = scene.meshes[inst.mesh].positions.astype(np.float64)
        if P.shape[0] != 642:  # the icospheres (subdivision 3)
            continue
        W = inst.world
        Q = P @ W[:3, :3].T + W[:3, 3]
        n = Q - W[:3, 3]
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        ro.append(Q + n * offset)
        rd.append(-n)
    return np.concatenate(ro).astype(np.float32), np.concatenate(rd).astype(np.float32)


def _cast(f, ro, rd):
    n = ro.shape[0]
    t = np.zeros(n, np.float32)
    tri = np.zeros(n, np.int32)
    inst = np.zeros(n, np.int32)
    _abi.check(f._lib.sb_raycast(f.ctx, _abi.ptr(ro), _abi.ptr(rd), n, _abi.ptr(t), _abi.ptr(tri), _abi.ptr(inst)),
               f.ctx)
    return t, tri, inst


def test_rays_through_shared_vertices_never_slip_through():
    s = synth.room_spheres(0)
    ro, rd = _vertex_rays(s)
    slips = {}
    for variant in (None, "watertight"):
        f = _field(s, variant)
        try:
            t, tri, inst = _cast(f, ro, rd)
        finally:
            f.dispose()
        occluded = (tri >= 0) & (t < 0.049)  # another sphere in front of this vertex
        hit_here = (tri >= 0) & (np.abs(t - 0.05) <= 1e-3)
        slips[variant or "mt"] = int((~occluded & ~hit_here).sum())
    print("rays through shared vertices:", ro.shape[0], "slipped through:", slips)
    assert slips["watertight"] == 0, slips


def test_watertight_hits_match_oracle_room():
    s = synth.room_spheres(0)
    f = _field(s, "watertight")
    try:
        mirror = gu.OracleMirror(f)
        rng = np.random.default_rng(11)
        n = 200_000
        ro = rng.uniform(0.3, 9.7, (n, 3)).astype(np.float32)
        rd = rng.normal(size=(n, 3))
        rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
        t, tri, inst = _cast(f, ro, rd)
        ot, otri, oinst, o2 = np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        orc.load().orc_closest(_abi.C.byref(mirror.scene), orc._p(ro), orc._p(rd), n, 1, 0, orc._p(ot),
                               orc._p(otri), orc._p(oinst), orc._p(o2), orc.threads())
        counts = gu.check_hits(mirror.scene, ro.astype(np.float64), rd.astype(np.float64), tri, inst, t, otri, oinst,
                               ot)
        print("watertight room raycast", counts)
    finally:
        f.dispose()


def test_watertight_atrium_solve_parity():
    s = synth.atrium(1)
    f = _field(s, "watertight")
    try:
        mirror = gu.OracleMirror(f)
        frame = f.tick()
        f.synchronize()
        r = gu.solve_parity(f, mirror, frame, f._params.to_array())
        print("watertight atrium solve", r)
        assert r["hit_share"] > 0.5
    finally:
        f.dispose()
