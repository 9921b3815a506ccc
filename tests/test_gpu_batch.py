"""The batched form (sb_solve_batch): several scenes and cascades through one
launch per stage give the same results as the same solves run one by one.

Two fields: the room-and-spheres scene (gated jitter, 1 directional + 4 point
lights) with an extra cascade twice its extent, and a 20k-triangle atrium
(clustered lights, montecarlo jitter, 48 rays). Three frames, each solving
the room's cascades 0 and 1 and the atrium's cascade 0; the batched run must
match the plain run bit for bit (hit records, histories and both atlases):
every item's arithmetic is the per-solve arithmetic.
"""
import numpy as np
import pytest

from speedball_b200 import _abi, synth
from speedball_b200.batch import BatchedFrame, GraphFrame, Lane, SolveItem, solveBatch

from gpu_util import make_field, read

pytestmark = pytest.mark.gpu

FRAMES = 3


def _fields():
    room = synth.room_spheres(0)
    a = make_field(room)
    g = room.meta["grid"]
    c1 = synth.nested_cascades(dict(g, rays=64), res=((8, 8, 8), (6, 6, 6)))[1]
    a.configureCascade(1, c1["gridMin"], c1["gridSize"], c1["res"])
    at = synth.atrium(seed=100, total_tris=20_000)
    at.meta["grid"] = dict(at.meta["grid"], res=(9, 9, 9), rays=48)
    at.meta["jitter"] = "montecarlo"
    b = make_field(at, rays=48)
    return a, b


def _state(f, ci):
    g = f.grid if ci == 0 else f._extraCascades[ci]
    P = g.res[0] * g.res[1] * g.res[2]
    n = P * g.raysPerProbe
    W, H = g.res[0] * 8, g.res[1] * g.res[2] * 8
    return dict(irr=read(f, "IRRADIANCE_HISTORY", P * 256, np.float32, ci),
                depth=read(f, "DEPTH_HISTORY", P * 128, np.float32, ci),
                atlas=read(f, "IRRADIANCE_ATLAS", W * H * 4, np.uint16, ci),
                datlas=read(f, "DEPTH_ATLAS", W * H * 4, np.uint16, ci),
                hits=read(f, "HIT_RECORDS", n * 4, np.uint32, ci),
                vis=read(f, "VISIBILITY", n * 4, np.uint32, ci))


def _run(batched: bool):
    a, b = _fields()
    fr = BatchedFrame([a, b], extra=[(a, 1)])
    for _ in range(FRAMES):
        if batched:
            fr.tick()
        else:
            fr.tickPlain()
    a.synchronize()
    b.synchronize()
    out = {"a0": _state(a, 0), "a1": _state(a, 1), "b0": _state(b, 0)}
    a.dispose()
    b.dispose()
    return out


def test_batched_solves_match_plain_bit_for_bit():
    plain = _run(False)
    batch = _run(True)
    for item in plain:
        for key in plain[item]:
            p, q = plain[item][key], batch[item][key]
            assert p.shape == q.shape
            bad = np.flatnonzero(p != q)
            assert bad.size == 0, (item, key, bad.size, bad[:8])
    # the frames did real work: lit texels and hits in every item
    for item in plain:
        assert (plain[item]["atlas"].view(np.float16)[0::4] > 0).any()
        assert (plain[item]["hits"][0::4] != 0xFFFFFFFF).any()


def _lanes(a, b):
    return [Lane(a, [(int(a.pool.blas_root[5]), int(a.pool.blas_end[5]))]),
            Lane(b, [(int(b.pool.blas_root[b._scene.meta["deformer"]]),
                      int(b.pool.blas_end[b._scene.meta["deformer"]]))])]


def _run_motion(graph: bool):
    a, b = _fields()
    fr = BatchedFrame([a, b], extra=[(a, 1)])
    lanes = _lanes(a, b)
    gf = GraphFrame(fr, lanes)
    for _ in range(FRAMES + 1):
        if graph:
            gf.tick()
        else:
            for l in lanes:
                for r, e in l.refits:
                    _abi.check(l.field._lib.sb_refit_blas(l.field.ctx, r, e), l.field.ctx)
                _abi.check(l.field._lib.sb_update_transforms(l.field.ctx, None, None, 0), l.field.ctx)
            fr.tick()
    a.synchronize()
    b.synchronize()
    out = {"a0": _state(a, 0), "a1": _state(a, 1), "b0": _state(b, 0),
           "nodes": read(b, "BVH_NODES", b.pool.bvhNodes.size, np.uint32)}
    gf.dispose()
    a.dispose()
    b.dispose()
    return out


def test_graph_frames_match_batched_frames():
    """The captured frame (motion lanes as parallel branches + batched solve),
    replayed with a new montecarlo jitter every frame, gives what the same
    frames give as ordinary launches."""
    ref = _run_motion(False)
    got = _run_motion(True)
    for item in ref:
        if item == "nodes":
            assert np.array_equal(ref[item], got[item])
            continue
        for key in ref[item]:
            bad = np.flatnonzero(ref[item][key] != got[item][key])
            assert bad.size == 0, (item, key, bad.size, bad[:8])


def test_batch_rejects_bad_items():
    a, b = _fields()
    try:
        with pytest.raises(_abi.SbError):
            solveBatch([SolveItem(a, 0, 0, 10), SolveItem(a, 0, 0, 10)])  # the same cascade twice
        with pytest.raises(_abi.SbError):
            solveBatch([SolveItem(a, 3, 0, 10)])  # cascade not configured
        with pytest.raises(_abi.SbError):
            solveBatch([SolveItem(b, 0, 0, 8)] * 17)
    finally:
        a.dispose()
        b.dispose()


def _solve_with_sort_key(key: int, frames: int = 4):
    import ctypes as C
    at = synth.atrium(seed=100, total_tris=20_000)
    at.meta["grid"] = dict(at.meta["grid"], res=(9, 9, 9), rays=48)
    f = make_field(at, rays=48)
    try:
        t = _abi.sb_tuning()
        _abi.check(f._lib.sb_get_tuning(f.ctx, C.byref(t)), f.ctx)
        t.sortKey = key
        _abi.check(f._lib.sb_set_tuning(f.ctx, C.byref(t)), f.ctx)
        for _ in range(frames):
            f.tick()
        f.synchronize()
        return _state(f, 0)
    finally:
        f.dispose()


def test_cost_ordered_issue_matches_tile_order():
    """sortKey 3 hands out the closest-hit batches costliest first (costs of
    the previous solve, ordered inside the shadow stage); every frame after
    the first runs in that order. Results do not depend on the issue order."""
    tile = _solve_with_sort_key(2)
    cost = _solve_with_sort_key(3)
    for key in tile:
        bad = np.flatnonzero(tile[key] != cost[key])
        assert bad.size == 0, (key, bad.size, bad[:8])
    assert (tile["hits"][0::4] != 0xFFFFFFFF).any()


def test_autotune_picks_a_candidate_and_restores_the_probes():
    from speedball_b200 import _abi as abi
    import ctypes as C
    f = make_field(synth.room_spheres(0))
    try:
        for _ in range(2):
            f.tick()
        f.synchronize()
        before = _state(f, 0)
        t = abi.sb_tuning()
        abi.check(f._lib.sb_autotune(f.ctx, 0, C.byref(t)), f.ctx)
        after = _state(f, 0)
        for key in ("irr", "depth", "atlas", "datlas"):
            assert np.array_equal(before[key], after[key]), key
        assert t.bvhKind in (0, 1, 2) and t.traceBlock in (128, 192, 256) and t.sortKey in (0, 1, 2, 3)
        assert t.smemWideNodes in (0, 73, 512)
        cur = abi.sb_tuning()
        abi.check(f._lib.sb_get_tuning(f.ctx, C.byref(cur)), f.ctx)
        assert (cur.traceBlock, cur.sortKey, cur.smemTlasNodes, cur.bvhKind) == \
               (t.traceBlock, t.sortKey, t.smemTlasNodes, t.bvhKind)
        f.tick()  # the tuned context keeps solving
        f.synchronize()
    finally:
        f.dispose()
