"""GPU parity on the paths a real frame takes: the atrium under the bench's
motion over feedback solves, montecarlo jitter epochs, partial updates with a
wrapping probe cursor and the normalised hysteresis exponent.

Each tick is checked three ways against the FP64 oracle:
  * the schedule: probe offset, probe count, jitter and hysteresis exponent
    equal the oracle's restatement of the reference's per-tick schedule
    (gi_probes.js:2947-2962, 3737-3788, 197-202, 235-251);
  * every ray of the solve: the GPU's hit triangle and instance equal the
    independent FP64 closest hit, or the oracle explains the difference ray by
    ray (near-tie within 1e-6 relative, or an FP32 edge graze / t order within
    the rounding bound of that ray's triangle test); hit t within 1e-5;
  * the oracle replays the GPU's hit and shadow decisions from its own state:
    every irradiance and depth texel within 1e-3 relative.
The scene state under motion (deformer refit, moved instance rows, TLAS refit)
is computed by the oracle and must equal the GPU's bit for bit.
"""
import numpy as np
import pytest

import orc
from speedball_b200 import synth

import gpu_util as gu

pytestmark = pytest.mark.gpu

IDX_JITTER = orc.ORC_PARAM_NAMES.index("frameJitter")
IDX_EXPONENT = orc.ORC_PARAM_NAMES.index("hysteresisExponent")


def _schedule_for(f, montecarlo: bool, normalize: bool) -> orc.Schedule:
    return orc.Schedule(f._probeTotal, f.getRays(), f._rayBudget, f._maxProbesPerTick, montecarlo, normalize)


def _tick(f, sched, now_ms):
    frame = f.tick(nowMs=now_ms)
    f.synchronize()
    want = sched.tick(now_ms)
    assert (frame["probeOffset"], frame["updatedCount"]) == (want["probeOffset"], want["updatedCount"])
    prm = f._params.to_array()
    assert prm[IDX_JITTER] == np.float32(want["frameJitter"]), (prm[IDX_JITTER], want["frameJitter"])
    assert prm[IDX_EXPONENT] == np.float32(want["hysteresisExponent"]), (prm[IDX_EXPONENT], want)
    return frame, prm, want


def _motion_parity(jitter: str, ticks: int = 4):
    s = synth.atrium(1)
    f = gu.make_field(s)
    try:
        if jitter == "montecarlo":
            f.setJitterMode("montecarlo")
        mirror = gu.OracleMirror(f)
        tail = gu.SceneTail(mirror)
        tail.check_gpu()
        sched = _schedule_for(f, jitter == "montecarlo", False)
        dm = s.meta["deformer"]
        report = []
        for k in range(ticks):
            mats, pos = synth.atrium_motion(s, k)
            s.meshes[dm].positions = pos
            for i, m in mats.items():
                s.instances[i].world = m
            f.markDeformsDirty()
            f.markTransformsDirty(list(mats))
            frame, prm, want = _tick(f, sched, 100.0 + 16.0 * k)
            assert frame["updatedCount"] == f._probeTotal
            tail.apply({dm: pos}, mats)
            tail.check_gpu()
            report.append(gu.solve_parity(f, mirror, frame, prm))
        assert report[-1]["lit"] > 0.05 and report[-1]["hit_share"] > 0.5
        return report
    finally:
        f.dispose()


@pytest.mark.parametrize("jitter", ["gated", "montecarlo"])
def test_atrium_motion_feedback_parity(jitter):
    """Config 1 as the bench runs it (deformer + 3 rigid movers every frame,
    full updates, clustered NEE) over 4 feedback solves; montecarlo advances
    the ray basis every solve."""
    report = _motion_parity(jitter)
    print(jitter, report)


def test_room_montecarlo_feedback_parity():
    """Room and spheres, montecarlo jitter over 5 solves: a new ray basis each
    solve, each checked against the oracle's directions for that epoch."""
    s = synth.room_spheres(0)
    f = gu.make_field(s)
    try:
        f.setJitterMode("montecarlo")
        mirror = gu.OracleMirror(f)
        sched = _schedule_for(f, True, False)
        jit = []
        for k in range(5):
            frame, prm, want = _tick(f, sched, 100.0 + 16.0 * k)
            jit.append(want["frameJitter"])
            r = gu.solve_parity(f, mirror, frame, prm)
        assert len(set(jit)) == 5 and all(0 < j < 1 for j in jit)
        assert r["lit"] > 0.05
    finally:
        f.dispose()


@pytest.mark.parametrize("case", ["room", "atrium"])
def test_partial_updates_parity(case):
    """The reference's per-tick path: a ray budget that covers part of the
    grid (room: 12,288 rays = 192 probes of 512; atrium: the default 98,304
    rays = 1,536 probes of 4,096), a probe cursor that wraps, and hysteresis
    normalisation on, so the exponent follows the service interval (ticks
    4 ms apart at 2.7 grid passes per revisit: exponent < 1)."""
    s = synth.room_spheres(0) if case == "room" else synth.atrium(1)
    f = gu.make_field(s)
    try:
        if case == "room":
            f.setRayBudget(12_288, maxProbesPerTick=2048)
        else:
            f.setRayBudget(98_304, maxProbesPerTick=2048)
        f.setHysteresisNormalization(True)
        mirror = gu.OracleMirror(f)
        sched = _schedule_for(f, False, True)
        ticks = 6 if case == "room" else 4
        offsets, exps = [], []
        for k in range(ticks):
            frame, prm, want = _tick(f, sched, 100.0 + 4.0 * k)
            offsets.append(frame["probeOffset"])
            exps.append(float(prm[IDX_EXPONENT]))
            assert frame["updatedCount"] < f._probeTotal
            gu.solve_parity(f, mirror, frame, prm)
        # the cursor wrapped past the end of the grid at least once, mid-solve
        assert any(o + frame["updatedCount"] > f._probeTotal for o in offsets)
        assert min(exps) < 1.0
    finally:
        f.dispose()


def test_fine_box_placement_matches_oracle():
    """fitFineBox on the GPU-resident pool equals the oracle's float64
    restatement bit for bit, and C1's resolution follows the reference's rule."""
    for s in (synth.atrium(1), synth.room_spheres(0), synth.atrium(3)):
        g = s.meta["grid"]
        f = gu.ProbeField(s, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=2,
                          rays=g["rays"], clusteredLighting=s.meta.get("clustered", False))
        try:
            pool = f.pool
            mn, size = f._c0Box
            box_size = [(mn[a] + size[a]) - mn[a] for a in range(3)]
            want = orc.fit_fine_box(pool.vertexData, pool.triIndex, mn, box_size)
            assert want is not None and f.hasFineCascade()
            got_min, got_size, got_box = f._c1Box
            assert got_box == box_size
            assert got_min == list(want[0]) and got_size == list(want[1]), (got_min, got_size, want)
            res = orc.fine_cascade_res(want[1], f._targetLongAxis, f._probeTotal)
            assert [f._c1Grid.res[a] for a in range(3)] == res
        finally:
            f.dispose()


def _tick2(f, sched, now_ms):
    frame = f.tick(nowMs=now_ms)
    f.synchronize()
    want = sched.tick(now_ms)
    got = frame["solves"]
    assert [(x["cascade"], x["probeOffset"], x["updatedCount"]) for x in got] == \
           [(w["cascade"], w["probeOffset"], w["updatedCount"]) for w in want]
    prms = []
    for x, w in zip(got, want):
        assert np.float32(x["hysteresisExponent"]) == np.float32(w["hysteresisExponent"]), (x, w)
        prm = f._params.to_array()
        prm[IDX_EXPONENT] = np.float32(w["hysteresisExponent"])
        assert prm[IDX_JITTER] == np.float32(w["frameJitter"])
        prms.append(prm)
    return got, prms


@pytest.mark.parametrize("budget", ["both", "alternating"])
def test_fine_cascade_parity(budget):
    """The atrium with its fitted fine cascade C1 (clustered NEE through C0's
    cell lists, each cascade's own bounce atlas): with a budget covering both
    cascades every tick solves C0 then C1; with the default 98,304-ray budget
    the cascades alternate with partial updates, and the exponent of a
    cascade's first solve falls back to twice the tick interval. Every solve
    is checked against the oracle (schedule, hit IDs ray by ray, texels)."""
    s = synth.atrium(1)
    g = s.meta["grid"]
    f = gu.ProbeField(s, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=2,
                      rays=g["rays"], clusteredLighting=True, hysteresis=s.meta["hysteresis"], recordHits=True)
    try:
        assert f.hasFineCascade()
        f.setHysteresisNormalization(True)
        if budget == "both":
            f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
        mirrors = [gu.OracleMirror(f, cascade=0), gu.OracleMirror(f, cascade=1)]
        sched = orc.Schedule2([f._probeTotal, f.cascadeProbes(1)], f.getRays(), f._rayBudget, f._maxProbesPerTick,
                              False, True)
        seen = set()
        for k in range(4):
            got, prms = _tick2(f, sched, 100.0 + 5.0 * k)
            for x, prm in zip(got, prms):
                seen.add(x["cascade"])
                gu.solve_parity(f, mirrors[x["cascade"]], x, prm)
        assert seen == {0, 1}
    finally:
        f.dispose()
