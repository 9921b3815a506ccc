"""The C-ABI library loads and exports every declared entry point; host-side
builders and host logic behave (CPU only, no device calls that need a GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from speedball_b200 import _abi
from speedball_b200 import field as fld
from speedball_b200 import scene as sc
from speedball_b200 import synth

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(sbh?_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_abi.SIGNATURES), set(names) - set(_abi.SIGNATURES)
    assert lib.sb_abi_version() == 3


def test_params_defaults_match_reference():
    p = _abi.default_params()
    assert p.hysteresis == pytest.approx(0.60)
    assert p.depthSharpness == 7.0 and p.radianceClamp == 8.0
    assert p.filterStrength == 1.0 and p.filterSmooth == 0.5
    assert p.tempChangeSigma1 == 2.5 and p.tempClampSigma == 6.0
    assert p.debugTempVarEps == pytest.approx(0.000025) and p.debugTempMinChangeH == pytest.approx(0.55)
    assert p.reflectionSkyFallback == 0.0 and p.skyConfigured == 0.0
    assert len(p.to_array()) == len(_abi.PARAM_NAMES) == 60


def test_params_vector_matches_oracle(orc):
    assert orc.load().orc_params_size() == len(_abi.PARAM_NAMES)


def test_null_arguments_rejected_without_device():
    lib = _abi.load()
    assert lib.sb_create(None, None) == _abi.SB_ERR_INVALID_ARG
    lib.sb_destroy(None)  # no-op
    assert lib.sb_synchronize(None) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_solve(None, 0, 0, 0) == _abi.SB_ERR_INVALID_ARG


def _check_threaded(nodes, n_tris, single=True):
    N = nodes.shape[0]
    seen = np.zeros(n_tris, int)
    for i in range(N):
        miss = int(nodes[i, 6])
        assert i < miss <= N
        if nodes[i, 7] == 0xFFFFFFFF:
            l, r = i + 1, int(nodes[i + 1, 6])
            assert l < r < miss or r == miss
            f = nodes.view(np.float32)
            assert (f[i, 0:3] <= np.minimum(f[l, 0:3], f[r, 0:3])).all()
        else:
            off, cnt = int(nodes[i, 7] & 0xFFFFFF), int(nodes[i, 7] >> 24)
            assert 1 <= cnt <= sc.MAX_LEAF and miss == i + 1
            seen[off:off + cnt] += 1
    assert (seen == 1).all()
    if single:
        assert nodes[0, 6] == N


def test_host_blas_builder_threaded_layout():
    P, F, _ = synth.icosphere(3)
    nodes, order = sc.build_blas(sc.Mesh(P, F, np.zeros(F.shape[0], np.uint32)))
    assert sorted(order.tolist()) == list(range(F.shape[0]))
    _check_threaded(nodes, F.shape[0])
    f = nodes.view(np.float32)
    # leaf bounds are exact
    for i in range(nodes.shape[0]):
        if nodes[i, 7] != 0xFFFFFFFF:
            off, cnt = int(nodes[i, 7] & 0xFFFFFF), int(nodes[i, 7] >> 24)
            V = P[F[order[off:off + cnt]].reshape(-1)]
            assert np.array_equal(f[i, 0:3], V.min(0)) and np.array_equal(f[i, 3:6], V.max(0))


def test_builder_degenerate_and_invalid():
    lib = _abi.load()
    P = np.zeros((3, 3), np.float32)
    F = np.tile(np.array([[0, 1, 2]], np.uint32), (40, 1))  # 40 coincident triangles
    nodes, order = sc.build_blas(sc.Mesh(P, F, np.zeros(40, np.uint32)))
    _check_threaded(nodes, 40)
    bad = np.array([[0, 1, 7]], np.uint32)
    out = np.zeros((2, 8), np.uint32)
    o = np.zeros(1, np.uint32)
    assert lib.sbh_build_blas(_abi.ptr(P), 3, _abi.ptr(bad), 1, 8, _abi.ptr(out), _abi.ptr(o)) == 0


def test_pool_assembly_room_spheres():
    s = synth.room_spheres(0)
    pool = sc.build_pool(s)
    assert pool.triIndex.shape[0] == 12 + 64 * 1280 == 81_932
    assert pool.instCount == 65 and pool.tlasNodeCount == sc.tlas_node_count(65)
    _check_threaded(pool.bvhNodes, pool.triIndex.shape[0], single=False)
    for m in range(len(s.meshes)):
        r, e = int(pool.blas_root[m]), int(pool.blas_end[m])
        assert pool.bvhNodes[r, 6] == e
        leaves = pool.bvhNodes[r:e][pool.bvhNodes[r:e, 7] != 0xFFFFFFFF, 7]
        offs = leaves & 0xFFFFFF
        assert offs.min() >= pool.tri_base[m] and offs.max() < pool.tri_base[m] + pool.tri_count[m]
        tri = pool.triIndex[pool.tri_base[m]:pool.tri_base[m] + pool.tri_count[m]]
        assert tri.min() >= pool.vert_base[m] and tri.max() < pool.vert_base[m] + pool.vert_count[m]
    assert pool.materials.shape[0] == pool.tlasBase + pool.tlasNodeCount * 12


def test_atrium_scale():
    s = synth.atrium(1)
    assert sum(m.indices.shape[0] for m in s.meshes) == 262_267
    assert len(s.meshes) == 30
    counts = [m.indices.shape[0] for m in s.meshes]
    assert min(counts) >= 500 and max(counts) <= 60_000
    assert s.lights.shape == (33, 17)
    assert len(s.meta["movers"]) == 3 and s.meta["deformer"] not in s.meta["movers"]


def test_tlas_node_count_formula(orc):
    lib = orc.load()
    for n in [1, 2, 3, 4, 5, 7, 30, 65, 400, 1000]:
        aabb = np.zeros((n, 9))
        aabb[:, 0:3] = np.arange(n)[:, None]
        aabb[:, 3:6] = aabb[:, 0:3] + 1
        aabb[:, 6:9] = aabb[:, 0:3] + 0.5
        tl = np.zeros((2 * n + 2, 12), np.float32)
        order = np.zeros(n, np.uint32)
        assert lib.orc_build_tlas(orc._p(aabb), n, orc._p(tl), orc._p(order), None) == sc.tlas_node_count(n)


def test_light_selection_and_scheduling():
    s = synth.atrium(1)
    recs, analytic, emitters = fld.selectGiLightRecords(s.lights, True, [0, 0, 0], [40, 20, 30])
    assert analytic == 33 and emitters == 0
    assert np.array_equal(recs, s.lights)  # fits the 64-record arena: original order
    many = np.concatenate([s.lights] * 3)
    recs2, a2, _ = fld.selectGiLightRecords(many, True, [0, 0, 0], [40, 20, 30])
    assert a2 == 64 and recs2[0][0] == 0  # directional lights rank first
    assert fld.probeUpdateIntervalTicks(4096, 1536) == pytest.approx(4096 / 1536)
    assert fld.hysteresisExponentForInterval(1000 / 120) == pytest.approx(0.5)
    assert fld.hysteresisExponentForInterval(100.0, False) == 1.0


def test_reflection_quality_resolution_and_abi_without_device():
    """resolveReflectionQuality (gi_probes.js:67-73): names in any case with
    surrounding space, the legacy boolean when no name is given (True = ultra),
    an unknown name rejected; the library refuses a tier above ultra and a null
    context before touching a device."""
    from speedball_b200.field import resolveReflectionQuality
    assert resolveReflectionQuality(None) == "off"
    assert resolveReflectionQuality(None, True) == "ultra"
    assert resolveReflectionQuality(" High ", True) == "high"
    assert resolveReflectionQuality("rough") == "rough"
    with pytest.raises(ValueError):
        resolveReflectionQuality("mirror")
    lib = _abi.load()
    assert lib.sb_set_reflection_quality(None, 1) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_get_reflection_layout(None, 0, None) == _abi.SB_ERR_INVALID_ARG
    prm = _abi.sb_gather_params()
    lib.sb_gather_params_defaults(C.byref(prm))
    assert prm.reflectionIntensity == 1.0 and prm.roughnessLimit == 1.0 and prm.cascades == 1
    assert lib.sb_gather_reflections(None, C.byref(prm), None, None, None, None, 0, None, None) == \
        _abi.SB_ERR_INVALID_ARG
    assert lib.sb_raycast_device(None, None, None, 0, None, None, None) == _abi.SB_ERR_INVALID_ARG
