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
    s.materials[::2, 4] = 1.0  # every other material fully metallic: no diffuse energy
    s.materials[::2, 7:10] = 0.0
    lay, reports, mirror = _run(s, "rough", 3)
    assert lay["tier"] == 1 and lay["glossyTile"] == 0
    print("rough room", reports[-1])
    cov = reports[-1]["rough_coverage_mean"]
    assert 0.2 < cov < 0.9, cov  # the metallic hits are left out of the lobe


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
