"""The update at the edges of its input space, each solve against the oracle as
in the other parity tests (hit IDs ray by ray, texels replayed within 1e-3):

  * the smallest grid (2 x 2 x 2 probes) at the fewest rays (32 per probe,
    gi_probes.js:988-992);
  * the most rays per probe (256: the blend stages them in four passes) and a
    ray count that is not a multiple of the 32-ray issue batches (48);
  * a full light arena of 64 point lights, unclustered, and clustered with
    every cell list overflowing its 16 slots (the all-lights fallback of
    gi_probes.js:2064-2127);
  * ragged partial updates: 13 probes from probe P - 5 (the range wraps, and
    the blend's 8-probe CTAs end mid-block), then 1 probe;
  * an update of 0 probes: accepted, nothing written.
"""
import numpy as np
import pytest

from speedball_b200 import _abi, synth
from speedball_b200.field import ProbeField

import gpu_util as gu

pytestmark = pytest.mark.gpu


def _field(scene, res, rays, clustered=False):
    g = scene.meta["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=res), cascades=1, rays=rays,
                   clusteredLighting=clustered, hysteresis=scene.meta.get("hysteresis"), jitterMode="gated",
                   recordHits=True)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
    return f


def _ticks(f, n):
    mirror = gu.OracleMirror(f)
    out = []
    for k in range(n):
        frame = f.tick(nowMs=100.0 + 16.0 * k)
        f.synchronize()
        out.append(gu.solve_parity(f, mirror, frame, f._params.to_array()))
    return out


@pytest.mark.parametrize("res,rays", [((2, 2, 2), 32), ((4, 4, 4), 256), ((5, 4, 3), 48)])
def test_grid_and_ray_extremes(res, rays):
    s = synth.room_spheres(0)
    f = _field(s, res, rays)
    try:
        assert f.getRays() == rays and f._probeTotal == res[0] * res[1] * res[2]
        r = _ticks(f, 2)
        print(res, rays, r[-1])
        assert r[-1]["lit"] > 0.0
    finally:
        f.dispose()


@pytest.mark.parametrize("clustered", [False, True])
def test_full_light_arena(clustered):
    s = synth.room_spheres(0, n_point=64, n_dir=0)
    f = _field(s, (6, 6, 6), 64, clustered)
    try:
        mirror = gu.OracleMirror(f)
        assert mirror.light_count == 64
        frame = f.tick(nowMs=100.0)
        f.synchronize()
        if clustered:
            # the cell lists (built before the first solve) equal the oracle's, and most
            # overflow (count 17): the emission falls back to all lights
            lights = gu.read(f, "LIGHTS", mirror.arena.shape[0], np.float32)
            cells = lights[64 * 17:].reshape(-1, 17)
            assert np.array_equal(cells, mirror.arena[64 * 17:].reshape(-1, 17))
            assert cells.shape[0] == 5 ** 3 and (cells[:, 0] == 17.0).mean() > 0.5
        r = gu.solve_parity(f, mirror, frame, f._params.to_array())
        print("clustered" if clustered else "all lights", r)
    finally:
        f.dispose()


def test_ragged_partial_updates_and_an_empty_one():
    s = synth.room_spheres(0)
    f = _field(s, (4, 4, 4), 64)
    try:
        P = f._probeTotal
        mirror = gu.OracleMirror(f)
        prm = f._params.to_array()
        _abi.check(f._lib.sb_set_params(f.ctx, _abi.C.byref(f._params)), f.ctx)
        for off, upd in ((P - 5, 13), (7, 1)):
            _abi.check(f._lib.sb_solve(f.ctx, 0, off, upd), f.ctx)
            f.synchronize()
            r = gu.solve_parity(f, mirror, dict(probeOffset=off, updatedCount=upd), prm)
            print(off, upd, r)
        before = gu.read(f, "IRRADIANCE_ATLAS", mirror.atlas.size, np.uint16)
        hist = gu.read(f, "IRRADIANCE_HISTORY", mirror.irr.size, np.float32)
        assert f._lib.sb_solve(f.ctx, 0, 3, 0) == _abi.SB_OK
        f.synchronize()
        assert np.array_equal(gu.read(f, "IRRADIANCE_ATLAS", mirror.atlas.size, np.uint16), before)
        assert np.array_equal(gu.read(f, "IRRADIANCE_HISTORY", mirror.irr.size, np.float32), hist)
    finally:
        f.dispose()
