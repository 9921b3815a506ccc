"""Failures injected from the host, each answered with a status and no GPU
fault, after which the context keeps working (the reference routes such
failures to onError or to a full rebuild: gi_probes.js:4170, 4220;
refitFlatBlasRange returning false, gi_refit.js:30-33).

  * a non-finite world matrix through sb_set_instances / sb_update_transforms:
    SB_ERR_INVALID_ARG before anything is enqueued;
  * a BLAS leaf whose triangle range leaves the pool, and an instance record
    whose BLAS range leaves the node pool, written by sb_upload_range: the next
    solve is refused on the device and sb_synchronize returns
    SB_ERR_LAYOUT_VIOLATION; writing the good words back recovers;
  * null host buffers: SB_ERR_INVALID_ARG;
  * the per-ray walk step limit run out on purpose (sb_set_walk_step_limit):
    every walk ends at the limit, sb_synchronize returns
    SB_ERR_DEVICE_WATCHDOG, and with the limit lifted the next solve is exact
    again;
  * a stale miss word that the reference's refit never reads: the refit still
    succeeds, bit-identical to the oracle's.
"""
import ctypes as C

import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu


@pytest.fixture()
def field():
    f = gu.make_field(synth.room_spheres(0))
    f.tick()
    f.synchronize()
    yield f
    f.dispose()


def _state(f):
    n = f._probeTotal * 256
    return gu.read(f, "IRRADIANCE_HISTORY", n, np.float32)


def _recovers(f):
    f.tick()
    assert f._lib.sb_synchronize(f.ctx) == _abi.SB_OK


def test_nonfinite_world_matrix_is_rejected(field):
    f = field
    lib, pool = f._lib, f.pool
    world = pool.inst_world.copy()
    world[5, 12] = np.nan
    st = lib.sb_set_instances(f.ctx, pool.instCount, _abi.ptr(world), _abi.ptr(pool.inst_active),
                              _abi.ptr(pool.inst_root), _abi.ptr(pool.inst_end))
    assert st == _abi.SB_ERR_INVALID_ARG
    src = np.array([3, 7], np.uint32)
    w2 = np.ascontiguousarray(pool.inst_world[[3, 7]].copy())
    w2[1, 0] = np.inf
    before = gu.read(f, "MATERIALS", pool.materials.shape[0], np.float32)
    assert lib.sb_update_transforms(f.ctx, _abi.ptr(src), _abi.ptr(w2), 2) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_synchronize(f.ctx) == _abi.SB_OK
    after = gu.read(f, "MATERIALS", pool.materials.shape[0], np.float32)
    assert np.array_equal(before.view(np.uint32), after.view(np.uint32))
    _recovers(f)


def test_out_of_range_leaf_is_a_layout_violation(field):
    f = field
    lib, pool = f._lib, f.pool
    r = int(pool.blas_root[9])
    seg = pool.bvhNodes[r:int(pool.blas_end[9])]
    leaf = r + int(np.flatnonzero(seg[:, 7] != 0xFFFFFFFF)[0])
    good = np.array([pool.bvhNodes[leaf, 7]], np.uint32)
    bad = np.array([(good[0] & 0xFF000000) | pool.triIndex.shape[0]], np.uint32)  # starts at triCount
    _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["BVH_NODES"], leaf * 8 + 7, 1, _abi.ptr(bad)), f.ctx)
    f.tick()
    assert lib.sb_synchronize(f.ctx) == _abi.SB_ERR_LAYOUT_VIOLATION
    _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["BVH_NODES"], leaf * 8 + 7, 1, _abi.ptr(good)), f.ctx)
    _recovers(f)


@pytest.mark.parametrize("word", [12, 13])
def test_out_of_range_instance_blas_range_is_a_layout_violation(field, word):
    f = field
    lib, pool = f._lib, f.pool
    at = pool.instBase + 4 * 28 + word  # slot 4: blasRoot (12) or blasEnd (13)
    good = gu.read(f, "MATERIALS", pool.materials.shape[0], np.float32)[at:at + 1].copy()
    bad = np.array([float(pool.bvhNodes.shape[0] + 5)], np.float32)
    _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["MATERIALS"], at, 1, _abi.ptr(bad)), f.ctx)
    f.tick()
    assert lib.sb_synchronize(f.ctx) == _abi.SB_ERR_LAYOUT_VIOLATION
    _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["MATERIALS"], at, 1, _abi.ptr(good)), f.ctx)
    _recovers(f)
    # the same range through the instance table is refused on the host
    ends = pool.inst_end.copy()
    ends[4] = pool.bvhNodes.shape[0] + 5
    assert lib.sb_set_instances(f.ctx, pool.instCount, _abi.ptr(pool.inst_world), _abi.ptr(pool.inst_active),
                                _abi.ptr(pool.inst_root), _abi.ptr(ends)) == _abi.SB_ERR_LAYOUT_VIOLATION


def test_null_buffers_are_invalid_arguments(field):
    f = field
    lib, pool = f._lib, f.pool
    assert lib.sb_upload_range(f.ctx, _abi.BUF["BVH_NODES"], 0, 8, None) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_set_instances(f.ctx, pool.instCount, None, _abi.ptr(pool.inst_active), _abi.ptr(pool.inst_root),
                                _abi.ptr(pool.inst_end)) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_update_transforms(f.ctx, None, _abi.ptr(pool.inst_world), 3) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_read_buffer(f.ctx, _abi.BUF["BVH_NODES"], 0, 8, None) == _abi.SB_ERR_INVALID_ARG
    _recovers(f)


@pytest.mark.parametrize("kind", [1, 2, 0])
def test_walk_step_limit_reports_watchdog(kind):
    """Every scene-BVH layout: a limit of 3 node steps ends every walk early and
    latches the watchdog; lifting it gives the solve of a context that never
    had it, bit for bit."""
    ref = gu.make_field(synth.room_spheres(0))
    f = gu.make_field(synth.room_spheres(0))
    try:
        for x in (ref, f):
            t = _abi.sb_tuning()
            _abi.check(x._lib.sb_get_tuning(x.ctx, C.byref(t)), x.ctx)
            t.bvhKind = kind
            _abi.check(x._lib.sb_set_tuning(x.ctx, C.byref(t)), x.ctx)
        lib = f._lib
        _abi.check(lib.sb_set_walk_step_limit(f.ctx, 3), f.ctx)
        f.tick()
        assert lib.sb_synchronize(f.ctx) == _abi.SB_ERR_DEVICE_WATCHDOG
        # the ray queries report it too
        ro = np.full((64, 3), 5.0, np.float32)
        rd = np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (64, 1))
        t = np.zeros(64, np.float32); tri = np.zeros(64, np.int32); inst = np.zeros(64, np.int32)
        st = lib.sb_raycast(f.ctx, _abi.ptr(ro), _abi.ptr(rd), 64, _abi.ptr(t), _abi.ptr(tri), _abi.ptr(inst))
        assert st == _abi.SB_ERR_DEVICE_WATCHDOG or lib.sb_synchronize(f.ctx) == _abi.SB_ERR_DEVICE_WATCHDOG
        _abi.check(lib.sb_set_walk_step_limit(f.ctx, 0), f.ctx)
        # clear the histories the truncated solve wrote, then both contexts solve once
        for x in (ref, f):
            P = x._probeTotal
            z = np.zeros(P * 256, np.float32)
            _abi.check(x._lib.sb_upload_range(x.ctx, _abi.BUF["IRRADIANCE_HISTORY"], 0, z.size, _abi.ptr(z)), x.ctx)
            _abi.check(x._lib.sb_upload_range(x.ctx, _abi.BUF["DEPTH_HISTORY"], 0, z.size // 2, _abi.ptr(z)), x.ctx)
            r = x.getResolution()
            a = np.zeros(r[0] * 8 * r[1] * r[2] * 8 * 4, np.uint16)
            a[3::4] = 0x3C00
            _abi.check(x._lib.sb_upload_range(x.ctx, _abi.BUF["IRRADIANCE_ATLAS"], 0, a.size, _abi.ptr(a)), x.ctx)
            _abi.check(x._lib.sb_upload_range(x.ctx, _abi.BUF["DEPTH_ATLAS"], 0, a.size, _abi.ptr(a)), x.ctx)
            x.tick()
            assert x._lib.sb_synchronize(x.ctx) == _abi.SB_OK
        assert np.array_equal(_state(f), _state(ref))
    finally:
        f.dispose()
        ref.dispose()


def test_stale_right_child_miss_word_refits_like_the_reference(field):
    """The reference's refit reads only left children's miss words
    (gi_refit.js:96-139), so a stale miss word on a right-child leaf leaves its
    refit valid. The CUDA refit then gives up its subtree partition (which
    trusts every miss word) and refits the range node by node: status OK and
    bounds bit-identical to the oracle's refit of the same words, on this call
    and the next."""
    f = field
    lib, pool = f._lib, f.pool
    m = 11
    r0, e0 = int(pool.blas_root[m]), int(pool.blas_end[m])
    nodes = pool.bvhNodes
    right = None
    for i in range(r0, e0 - 1):
        if nodes[i, 7] == 0xFFFFFFFF:
            r = int(nodes[i + 1, 6])
            if nodes[r, 7] != 0xFFFFFFFF and r + 2 <= e0:
                right = r
                break
    assert right is not None
    stale = np.array([right + 2], np.uint32)
    _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["BVH_NODES"], right * 8 + 6, 1, _abi.ptr(stale)), f.ctx)
    vd = pool.vertexData.copy()
    vb, vc = int(pool.vert_base[m]), int(pool.vert_count[m])
    rng = np.random.default_rng(21)
    want = gu.read(f, "BVH_NODES", nodes.size, np.uint32).reshape(-1, 8)
    for _ in range(2):
        vd[vb:vb + vc, 0:3] += rng.normal(0, 0.05, (vc, 3)).astype(np.float32)
        sl = np.ascontiguousarray(vd[vb:vb + vc])
        _abi.check(lib.sb_update_deform(f.ctx, vb, vc, _abi.ptr(sl), r0, e0), f.ctx)
        assert lib.sb_synchronize(f.ctx) == _abi.SB_OK
        got = gu.read(f, "BVH_NODES", nodes.size, np.uint32).reshape(-1, 8)
        assert orc.load().orc_refit_blas(orc._p(want), want.size, orc._p(pool.triIndex), pool.triIndex.size,
                                         orc._p(vd), vd.size, r0, e0) == 1
        assert np.array_equal(got[r0:e0], want[r0:e0])
