"""Background scene-BVH builds (sb_set_scene_bvh_build_mode) on the atrium
under the bench's motion, every solve checked against the FP64 oracle as in
tests/test_gpu_schedules.py (hit IDs ray by ray, texels replayed within 1e-3):

  * the first tick starts the build on a host thread and is answered by the
    reference's two-level walk (GPU-refit TLAS + BLASes);
  * the deformer and the three movers move while the build runs: the tree,
    built from the placements read at its start, is installed with those slots
    marked, so the solves after it stay on the oracle's answer;
  * a structural change while a build runs drops that build; the next tick
    starts a new one, which is installed.
"""
import numpy as np
import pytest

import orc
from speedball_b200 import synth

import gpu_util as gu

pytestmark = pytest.mark.gpu


def test_background_build_under_motion_matches_oracle():
    s = synth.atrium(1)
    f = gu.make_field(s, sceneBvhBuild="background")
    try:
        mirror = gu.OracleMirror(f)
        tail = gu.SceneTail(mirror)
        sched = orc.Schedule(f._probeTotal, f.getRays(), f._rayBudget, f._maxProbesPerTick, False, False)
        dm = s.meta["deformer"]
        report = []

        def frame(k):
            mats, pos = synth.atrium_motion(s, k)
            s.meshes[dm].positions = pos
            for i, m in mats.items():
                s.instances[i].world = m
            f.markDeformsDirty()
            f.markTransformsDirty(list(mats))
            now = 100.0 + 16.0 * k
            fr = f.tick(nowMs=now)
            f.synchronize()
            want = sched.tick(now)
            assert (fr["probeOffset"], fr["updatedCount"]) == (want["probeOffset"], want["updatedCount"])
            tail.apply({dm: pos}, mats)
            tail.check_gpu()
            r = gu.solve_parity(f, mirror, fr, f._params.to_array())
            report.append(r)
            return f.getStats()

        st = frame(0)  # the build starts here; the two-level walk answers
        assert st["sceneBvhBuilding"] and not st["sceneBvhActive"] and st["sceneBvhBuilds"] == 0, st
        st = frame(1)  # the movers and the deformer move while it runs (or it is installed here)
        f.finishSceneBvh()
        st = f.getStats()
        assert st["sceneBvhActive"] and not st["sceneBvhBuilding"] and st["sceneBvhBuilds"] == 1, st
        for k in (2, 3):  # the installed tree, with the moved slots walked through their BLASes
            st = frame(k)
            assert st["sceneBvhActive"], st

        # a structural change during a build drops it
        f.rebuildSceneBvh()
        st = frame(4)  # starts build 2
        assert st["sceneBvhBuilding"] and not st["sceneBvhActive"], st
        f.rebuildSceneBvh()
        f.finishSceneBvh()  # build 2 predates the change: dropped
        st = f.getStats()
        assert not st["sceneBvhActive"] and not st["sceneBvhBuilding"] and st["sceneBvhBuilds"] == 1, st
        st = frame(5)  # starts build 3
        assert st["sceneBvhBuilding"], st
        f.finishSceneBvh()
        st = frame(6)
        assert st["sceneBvhActive"] and st["sceneBvhBuilds"] == 2, st
        print(report)
        assert report[-1]["lit"] > 0.05 and report[-1]["hit_share"] > 0.5
    finally:
        f.dispose()


def test_build_mode_argument_checked():
    s = synth.room_spheres(0)
    f = gu.make_field(s)
    try:
        from speedball_b200 import _abi
        assert f._lib.sb_set_scene_bvh_build_mode(f.ctx, 2) == _abi.SB_ERR_INVALID_ARG
        assert f._lib.sb_finish_scene_bvh(f.ctx) == _abi.SB_OK  # nothing running: a no-op
        with pytest.raises(ValueError):
            f.setSceneBvhBuild("lazy")
    finally:
        f.dispose()


def test_dispose_and_layout_change_while_building():
    """A context destroyed while its background build runs waits for the build
    and frees it; a layout change (bvhKind) during a build drops it, and the
    next tick builds the new layout's trees."""
    import ctypes as C
    s = synth.atrium(1)
    f = gu.make_field(s, sceneBvhBuild="background")
    f.tick(nowMs=100.0)
    assert f.getStats()["sceneBvhBuilding"]
    f.dispose()  # joins the build thread

    f = gu.make_field(s, sceneBvhBuild="background")
    try:
        f.tick(nowMs=100.0)
        assert f.getStats()["sceneBvhBuilding"]
        from speedball_b200 import _abi
        t = _abi.sb_tuning()
        _abi.check(f._lib.sb_get_tuning(f.ctx, C.byref(t)), f.ctx)
        t.bvhKind = 2  # binary only: a structural change for the scene BVH
        _abi.check(f._lib.sb_set_tuning(f.ctx, C.byref(t)), f.ctx)
        f.finishSceneBvh()  # the build of the 8-wide layout is dropped
        st = f.getStats()
        assert not st["sceneBvhActive"] and st["sceneBvhBuilds"] == 0, st
        f.tick(nowMs=116.0)  # starts the binary-only build
        f.finishSceneBvh()
        f.tick(nowMs=132.0)
        f.synchronize()
        st = f.getStats()
        assert st["sceneBvhActive"] and st["sceneBvhBuilds"] == 1, st
    finally:
        f.dispose()


def test_blocking_mode_waits_for_a_running_build():
    """Switched back to blocking mode while a background build runs: the next
    tick waits for that build and traces with the new tree."""
    s = synth.atrium(1)
    f = gu.make_field(s, sceneBvhBuild="background")
    try:
        f.tick(nowMs=100.0)
        assert f.getStats()["sceneBvhBuilding"]
        f.setSceneBvhBuild("blocking")
        f.tick(nowMs=116.0)
        f.synchronize()
        st = f.getStats()
        assert st["sceneBvhActive"] and not st["sceneBvhBuilding"] and st["sceneBvhBuilds"] == 1, st
    finally:
        f.dispose()
