"""Reflection lobes (reflectionQuality rough / high / ultra, gi_probes.js:60-75)
on the GPU against the oracle.

  * room + 64 spheres, tier rough: every other material fully metallic, so
    about half the hits are stored as -(t + 2) (gi_probes.js:2055-2062) and
    left out of the power-8 lobe; 3 feedback solves;
  * atrium (open above), tiers high and ultra with a configured sky and the
    sky fallback on, so misses feed the lobes: the power-64 glossy tiles, the
    high tier's two texel phases over 4 solves, partial updates with a
    wrapping cursor for high;
every solve checked as the other parity tests check it (schedule, hit IDs ray
by ray, irradiance and depth texels replayed by the oracle), plus the rough
history and atlas and the glossy numerator, support and atlas within 1e-3 of
the oracle's replay, and the glossy phase. Batched solves and the adjoint
refuse the lobes (SB_ERR_UNSUPPORTED).
"""
import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu

SKY = np.array([[1.0, 1.1, 1.3], [0.1, 0.12, 0.2], [0.3, 0.3, 0.35], [0.05, 0.04, 0.02]] + [[0.0, 0.0, 0.0]] * 5,
               np.float32)


def _run(scene, tier, solves, budget=None, sky=False):
    f = gu.make_field(scene, reflectionQuality=tier, reflectionSkyFallback=sky)
    try:
        if sky:
            f.setSky(SKY)
        if budget:
            f.setRayBudget(budget, maxProbesPerTick=2048)
        lay = f.reflectionLayout(0)
        mirror = gu.OracleMirror(f)
        sched = orc.Schedule(f._probeTotal, f.getRays(), f._rayBudget, f._maxProbesPerTick, False, False)
        reports = []
        for k in range(solves):
            frame = f.tick(nowMs=100.0 + 16.0 * k)
            f.synchronize()
            want = sched.tick(100.0 + 16.0 * k)
            assert (frame["probeOffset"], frame["updatedCount"]) == (want["probeOffset"], want["updatedCount"])
            reports.append(gu.solve_parity(f, mirror, frame, f._params.to_array()))
        return lay, reports, mirror
    finally:
        f.dispose()


def test_rough_tier_room_with_metals():
    s = synth.room_spheres(0)
    s.materials = s.materials.copy()
    walls = int(s.meshes[0].tri_material[0])
    metal = [m for m in range(0, s.materials.shape[0], 2) if m != walls]
    s.materials[metal, 4] = 1.0  # every other sphere material fully metallic: no diffuse energy
    s.materials[metal, 7:10] = 0.0
    lay, reports, mirror = _run(s, "rough", 3)
    assert lay["tier"] == 1 and lay["glossyTile"] == 0
    print("rough room", reports[-1])
    cov = reports[-1]["rough_coverage_mean"]
    assert 0.3 < cov < 0.999, cov  # the metallic hits are left out of the lobe


@pytest.mark.parametrize("tier", ["high", "ultra"])
def test_glossy_tiers_atrium_with_sky(tier):
    s = synth.atrium(1)
    budget = 98_304 if tier == "high" else None  # high: partial updates, the cursor wraps
    lay, reports, mirror = _run(s, tier, 4, budget=budget, sky=True)
    want_tile = 10 if tier == "high" else 18
    assert (lay["glossyTile"], lay["glossyTilesX"], lay["glossyTilesY"]) == (want_tile, 64, 64)
    assert lay["glossyAtlasW"] == 64 * want_tile
    print(tier, reports[-1])
    assert reports[-1]["hit_share"] < 0.95  # some rays reach the sky and count through the fallback
    den = mirror.rf.glossy_den.reshape(-1, want_tile * want_tile)
    assert (den > 0).mean() > 0.5


def test_reflection_tiers_refuse_batch_and_adjoint():
    s = synth.room_spheres(0)
    f = gu.make_field(s, reflectionQuality="rough")
    try:
        items = (_abi.sb_solve_item * 1)()
        items[0].ctx = f.ctx
        items[0].cascade = 0
        items[0].probeOffset = 0
        items[0].updatedCount = f._probeTotal
        assert f._lib.sb_solve_batch(items, 1) == _abi.SB_ERR_UNSUPPORTED
        loss = _abi.C.c_double(0.0)
        assert f._lib.sb_forward_record(f.ctx, 0, 1, None, _abi.C.byref(loss)) == _abi.SB_ERR_UNSUPPORTED
        assert f._lib.sb_set_reflection_quality(f.ctx, 4) == _abi.SB_ERR_INVALID_ARG
        # switching the tier off frees the lobes; the plain path runs
        assert f._lib.sb_set_reflection_quality(f.ctx, 0) == _abi.SB_OK
        assert f.reflectionLayout(0)["tier"] == 0
        f.tick()
        f.synchronize()
    finally:
        f.dispose()


def _reflect_atlases(f, ci):
    g = f.cascadeGrid(ci)
    r = [g.res[a] for a in range(3)]
    W, H = r[0] * 8, r[1] * r[2] * 8
    a = gu.read(f, "IRRADIANCE_ATLAS", W * H * 4, np.uint16, ci)
    d = gu.read(f, "DEPTH_ATLAS", W * H * 4, np.uint16, ci)
    rough = gu.read(f, "ROUGH_ATLAS", W * H * 4, np.uint16, ci)
    lay = f.reflectionLayout(ci)
    glossy = None
    if lay["glossyTile"]:
        glossy = gu.read(f, "GLOSSY_ATLAS", lay["glossyAtlasW"] * lay["glossyAtlasH"] * 4, np.uint16, ci)
        glossy = glossy.reshape(lay["glossyAtlasH"], lay["glossyAtlasW"], 4)
    ra = orc.reflect_atlas(rough, glossy, lay["glossyOct"], lay["glossyTilesX"])
    return orc.grid_struct(gu.grid_dict(g)), a, d, ra


@pytest.mark.parametrize("case", ["one_cascade", "two_cascades_chebyshev"])
def test_combined_receiver_matches_oracle(case):
    """sb_gather_reflections on the atlases of 4 solves (room with metals, tier
    high, a fine box as cascade 1): irradiance and the reflection layer of
    200,000 receivers (roughness uniform in [0, 1], limit 0.9, intensity 0.8)
    within 1e-3 of the FP64 combined receiver; samples within 1e-4 of a
    discontinuity (cage floor, Chebyshev select, parallax root selects, the
    roughness limit) are counted, must be rare, and are not compared."""
    torch = pytest.importorskip("torch")
    s = synth.room_spheres(0)
    s.materials = s.materials.copy()
    walls = int(s.meshes[0].tri_material[0])
    s.materials[[m for m in range(0, s.materials.shape[0], 2) if m != walls], 4] = 1.0
    f = gu.make_field(s, reflectionQuality="high")
    try:
        g = s.meta["grid"]
        gmin = np.asarray(g["gridMin"], np.float64)
        gsz = np.asarray(g["gridSize"], np.float64)
        f.configureCascade(1, (gmin + gsz * 0.25).tolist(), (gsz * 0.5).tolist(), (8, 8, 8))
        for _ in range(4):
            fr = f.beginTick()
            _abi.check(f._lib.sb_solve(f.ctx, 0, fr["probeOffset"], fr["updatedCount"]), f.ctx)
            _abi.check(f._lib.sb_solve(f.ctx, 1, 0, f.cascadeProbes(1)), f.ctx)
            f.endTick(fr)
        f.synchronize()
        n = 200_000
        rng = np.random.default_rng(9)
        lo = gmin - 0.1
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = rng.uniform(lo, lo + gsz + 0.2, (n, 3))
        nv = rng.normal(size=(n, 3))
        nv /= np.linalg.norm(nv, axis=1, keepdims=True)
        a4 = np.zeros((n, 4), np.float32); a4[:, :3] = nv
        rd = rng.normal(size=(n, 3))
        rd /= np.linalg.norm(rd, axis=1, keepdims=True)
        r4 = np.zeros((n, 4), np.float32); r4[:, :3] = rd; r4[:, 3] = rng.uniform(0, 1, n)
        two = case != "one_cascade"
        kw = dict(reflectionIntensity=0.8, roughnessLimit=0.9)
        if two:
            kw.update(cascades=2.0, chebyStrength=1.0, chebyBias0=0.02, chebyBias1=0.01, borderBand=0.2)
        prm = _abi.sb_gather_params()
        f._lib.sb_gather_params_defaults(_abi.C.byref(prm))
        prm.reflectionIntensity, prm.roughnessLimit = 0.8, 0.9
        if two:
            prm.cascades, prm.chebyStrength, prm.borderBand = 2, 1.0, 0.2
            prm.chebyBias[0], prm.chebyBias[1] = 0.02, 0.01
        dev = torch.device("cuda", 0)
        tp, tn, tr = (torch.from_numpy(x).to(dev) for x in (pos, a4, r4))
        oi = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        orf = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        _abi.check(f._lib.sb_gather_reflections(f.ctx, _abi.C.byref(prm), tp.data_ptr(), tn.data_ptr(), tn.data_ptr(),
                                                tr.data_ptr(), n, oi.data_ptr(), orf.data_ptr()), f.ctx)
        f.synchronize()
        gi, gr = oi.cpu().numpy(), orf.cpu().numpy()
        G0, a0, d0, r0 = _reflect_atlases(f, 0)
        G1, a1, d1, r1 = _reflect_atlases(f, 1)
        wi, wr, near = orc.gather_combined(G0, a0, d0, r0, orc.gather_params(**kw), pos, a4, a4, r4,
                                           G1 if two else None, a1 if two else None, d1 if two else None,
                                           r1 if two else None)
        edge = near < 1e-4
        assert edge.mean() < 5e-3, edge.mean()
        ei = gu.texel_rel_err(gi[~edge, :3].astype(np.float64), wi[~edge])
        er = gu.texel_rel_err(gr[~edge, :3].astype(np.float64), wr[~edge, :3])
        ec = gu.texel_rel_err(gr[~edge, 3].astype(np.float64), wr[~edge, 3])
        print(case, "irr", ei.max(), "refl", er.max(), "coverage", ec.max(), "edge", int(edge.sum()),
              "covered share", float((wr[:, 3] > 0).mean()))
        keep = np.flatnonzero(~edge)
        for name, e, gv, ov in (("refl", er.max(1), gr[keep, :3], wr[keep, :3]), ("coverage", ec, gr[keep, 3], wr[keep, 3])):
            worst = np.argsort(e)[-5:]
            print(name, "abs err max", float(np.abs(gv.astype(np.float64) - ov).max()), "scale", float(np.abs(ov).max()),
                  "over 1e-3:", int((e > 1e-3).sum()),
                  [(float(e[k]), np.asarray(gv[k]).tolist(), np.asarray(ov[k]).tolist(), float(r4[keep[k], 3]),
                    float(near[keep[k]])) for k in worst])
        assert max(ei.max(), er.max(), ec.max()) <= gu.TEXEL_REL
        assert (wr[:, 3] > 0).mean() > 0.5 and wr[:, :3].max() > 0.01
        assert lib_refuses_without_lobes(f)
    finally:
        f.dispose()


def lib_refuses_without_lobes(f) -> bool:
    prm = _abi.sb_gather_params()
    f._lib.sb_gather_params_defaults(_abi.C.byref(prm))
    _abi.check(f._lib.sb_set_reflection_quality(f.ctx, 0), f.ctx)
    torch = pytest.importorskip("torch")
    buf = torch.zeros((64, 4), dtype=torch.float32, device=torch.device("cuda", 0))
    p = buf.data_ptr()
    return f._lib.sb_gather_reflections(f.ctx, _abi.C.byref(prm), p, p, p, p, 8, p, p) == _abi.SB_ERR_NOT_READY


@pytest.mark.parametrize("tier", ["rough", "ultra"])
def test_reflection_lobes_with_emitters(tier):
    """giEmitter virtual rays enter the rough lobe (power-8 secondary weight)
    and the glossy lobe (power 64) as well as the diffuse moments
    (gi_probes.js:2262-2310, 2624-2638): the room with one sphere and two
    point emitters, montecarlo ticks, every lobe against the oracle given the
    GPU's emitter visibility history."""
    s = synth.add_emitters(synth.room_spheres(0))
    f = gu.make_field(s, reflectionQuality=tier)
    try:
        f.setJitterMode("montecarlo")
        mirror = gu.OracleMirror(f)
        assert mirror.emitters == (5, 3)
        for k in range(3):
            frame = f.tick(nowMs=100.0 + 16.0 * k)
            f.synchronize()
            r = gu.solve_parity(f, mirror, frame, f._params.to_array())
            print(tier, k, {key: r[key] for key in r if "err" in key or "agreement" in key})
    finally:
        f.dispose()


def test_captured_frame_refuses_lobes_set_after_capture():
    """A frame graph captured without lobes does not replay once a tier is set:
    the batched kernels have no lobes, so the replay (and its re-capture) return
    SB_ERR_UNSUPPORTED instead of leaving the lobes unwritten."""
    s = synth.room_spheres(0)
    f = gu.make_field(s)
    try:
        fr = f.beginTick()
        _abi.check(f._lib.sb_graph_capture_frame(f.ctx, 0, fr["probeOffset"], fr["updatedCount"], None, None, 0, 0),
                   f.ctx)
        f.endTick(fr)
        _abi.check(f._lib.sb_graph_launch(f.ctx), f.ctx)
        f.synchronize()
        _abi.check(f._lib.sb_set_reflection_quality(f.ctx, 1), f.ctx)
        assert f._lib.sb_graph_launch(f.ctx) == _abi.SB_ERR_UNSUPPORTED
        _abi.check(f._lib.sb_graph_destroy(f.ctx), f.ctx)
    finally:
        f.dispose()
