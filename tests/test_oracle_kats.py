"""Known-answer and property tests of the oracle (CPU, no GPU).

The reference ships no golden vectors for this path (its oct round-trip test
scripts/gi-oct-test.mjs and the refit smoke tests are absent), so these pin the
restatement against the reference's own stated invariants (gi_oct.js:15-19,
gi_refit.js:10-33, 298-346) and against independent computations.
"""
import ctypes as C
import math

import numpy as np
import pytest

from speedball_b200 import scene as sc
from speedball_b200 import synth


def _v(n):
    return (C.c_double * n)()


def test_oct_roundtrip_and_seam(orc):
    lib = orc.load()
    rng = np.random.default_rng(0)
    for _ in range(2000):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        uv, d = _v(2), _v(3)
        lib.orc_oct_encode((C.c_double * 3)(*n), uv)
        assert 0.0 <= uv[0] <= 1.0 and 0.0 <= uv[1] <= 1.0
        lib.orc_oct_decode(uv, d)
        assert np.allclose(np.array(d[:]), n, atol=1e-12)
    # opposite tile edges map to antipodal-mirrored directions (gi_oct.js:15-19)
    for t in np.linspace(0.0, 1.0, 33):
        a, b = _v(3), _v(3)
        lib.orc_oct_decode((C.c_double * 2)(0.0, t), a)
        lib.orc_oct_decode((C.c_double * 2)(0.0, 1.0 - t), b)
        assert a[2] <= 1e-12 and abs(a[0] - b[0]) < 1e-12 and abs(a[1] + b[1]) < 1e-12 and abs(a[2] - b[2]) < 1e-12


def test_to_half_matches_ieee(orc):
    lib = orc.load()
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.normal(size=4000) * 10 ** rng.uniform(-9, 5, 4000),
                           [0.0, -0.0, 65504.0, 65520.0, 1e-8, 2 ** -24, 2 ** -25, 3 * 2 ** -26, 1.0, 0.5]])
    for v in vals:
        h = lib.orc_to_half(float(v))
        ref = np.array([v], np.float64).astype(np.float16).view(np.uint16)[0]
        assert h == ref, (v, hex(h), hex(ref))
        if not math.isinf(float(np.float16(v))):
            assert lib.orc_from_half(h) == float(np.float16(v))


def test_ray_dir_gated_fibonacci(orc):
    lib = orc.load()
    N = 64
    d = _v(3)
    for k in range(N):
        lib.orc_ray_dir(k, N, 0.0, d)
        v = np.array(d[:])
        assert abs(np.linalg.norm(v) - 1) < 1e-12
        assert abs(v[2] - (1 - 2 * (k + 0.5) / N)) < 1e-12
        phi = k * math.pi * (3 - math.sqrt(5))
        r = math.sqrt(1 - v[2] ** 2)
        assert abs(v[0] - r * math.cos(phi)) < 1e-12 and abs(v[1] - r * math.sin(phi)) < 1e-12


def test_hysteresis_exponent(orc):
    lib = orc.load()
    ref = 1000 / 60
    assert lib.orc_hysteresis_exponent(5.0, 0) == 1.0
    assert abs(lib.orc_hysteresis_exponent(ref / 2, 1) - 0.5) < 1e-15
    assert lib.orc_hysteresis_exponent(ref * 3, 1) == 1.0
    assert lib.orc_hysteresis_exponent(float("nan"), 1) == 1.0
    assert lib.orc_hysteresis_exponent(-3, 1) == 0.0


def test_grid_resolution(orc):
    from speedball_b200.field import computeGridResolution
    lib = orc.load()
    for size, target in [((10, 10, 10), 8), ((40, 20, 30), 16), ((1, 100, 3), 12), ((0.0, 0, 0), 12)]:
        out = (C.c_uint32 * 3)()
        lib.orc_grid_resolution((C.c_double * 3)(*size), target, out)
        assert tuple(out) == computeGridResolution(size, target)
    out = (C.c_uint32 * 3)()
    lib.orc_grid_resolution((C.c_double * 3)(10 * 1.12, 10 * 1.12, 10 * 1.12), 8, out)
    assert tuple(out) == (9, 9, 9)  # divisions=8 on a padded cube gives 9^3 probes


def test_gutter_is_canonical_mirror(orc):
    lib = orc.load()
    src = [lib.orc_gutter_source_lane(l) for l in range(64)]
    for l in range(64):
        lx, ly = l % 8, l // 8
        s = src[l]
        sx, sy = s % 6 + 1, s // 6 + 1
        if 1 <= lx <= 6 and 1 <= ly <= 6:
            assert (sx, sy) == (lx, ly)
        elif lx in (0, 7) and ly in (0, 7):
            assert (sx, sy) == ((6 if lx == 0 else 1), (6 if ly == 0 else 1))
        elif ly in (0, 7):
            assert (sx, sy) == (7 - lx, 1 if ly == 0 else 6)
        else:
            assert (sx, sy) == (1 if lx == 0 else 6, 7 - ly)


@pytest.fixture(scope="module")
def room(orc):
    s = synth.room_spheres(0)
    pool = sc.build_pool(s)
    mats, order, live, aabb = orc.compute_tail(pool)
    return s, pool, mats, order, live, aabb


def test_tlas_build_invariants(orc, room):
    s, pool, mats, order, live, aabb = room
    assert sorted(order.tolist()) == list(range(pool.instCount))
    tl = mats[pool.tlasBase:].reshape(-1, 12)
    n = tl.shape[0]
    assert n == pool.tlasNodeCount
    owner = np.full(pool.instCount, -1)
    for i in range(n):
        if tl[i, 8] > 0:
            off, cnt = int(tl[i, 7]), int(tl[i, 8])
            assert 1 <= cnt <= 2 and tl[i, 6] == i + 1
            owner[off:off + cnt] = i
            # leaf bounds are the f32 union of its slots
            assert np.array_equal(tl[i, 0:3], live[off:off + cnt, 0:3].min(0))
            assert np.array_equal(tl[i, 3:6], live[off:off + cnt, 3:6].max(0))
        else:
            l, r = i + 1, int(tl[i + 1, 6])
            assert l < r < n
            assert np.array_equal(tl[i, 0:3], np.minimum(tl[l, 0:3], tl[r, 0:3]))
            assert np.array_equal(tl[i, 3:6], np.maximum(tl[l, 3:6], tl[r, 3:6]))
    assert (owner >= 0).all()
    assert tl[0, 6] == n


def test_tlas_refit_range_and_dirty_agree(orc, room):
    s, pool, mats, order, live, aabb = room
    lib = orc.load()
    rng = np.random.default_rng(3)
    tl0 = np.ascontiguousarray(mats[pool.tlasBase:].reshape(-1, 12))
    live2 = live.copy()
    dirty = np.sort(rng.choice(pool.instCount, 7, replace=False)).astype(np.uint32)
    live2[dirty] += rng.uniform(-0.5, 0.5, (7, 6)).astype(np.float32)
    live2[dirty, 3:6] = np.maximum(live2[dirty, 3:6], live2[dirty, 0:3])
    a, b = tl0.copy(), tl0.copy()
    assert lib.orc_refit_tlas_range(orc._p(a), a.size, orc._p(live2), live2.size, 0, a.shape[0]) == 1
    touched = np.zeros(a.shape[0], np.uint32)
    cnt = C.c_uint32()
    assert lib.orc_refit_tlas_dirty(orc._p(b), b.size, orc._p(live2), live2.size, b.shape[0], orc._p(dirty),
                                    dirty.size, orc._p(touched), C.byref(cnt)) == 1
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert 0 in touched[:cnt.value].tolist()
    # a corrupt miss link fails closed (gi_refit.js:275)
    c = tl0.copy()
    interior = [i for i in range(c.shape[0]) if c[i, 8] == 0]
    c[interior[0] + 1, 6] = 0.5
    assert lib.orc_refit_tlas_range(orc._p(c), c.size, orc._p(live2), live2.size, 0, c.shape[0]) == 0


def test_blas_refit_exact(orc, room):
    s, pool, mats, order, live, aabb = room
    lib = orc.load()
    nodes = pool.bvhNodes.copy()
    vd = pool.vertexData.copy()
    # unmodified geometry: refit reproduces the builder's exact bounds
    r, e = int(pool.blas_root[5]), int(pool.blas_end[5])
    n2 = nodes.copy()
    assert lib.orc_refit_blas(orc._p(n2), n2.size, orc._p(pool.triIndex), pool.triIndex.size, orc._p(vd), vd.size, r, e)
    assert np.array_equal(n2, nodes)
    # deform and check leaves are exact min/max of their triangles, interiors the union
    v0, vc = int(pool.vert_base[5]), int(pool.vert_count[5])
    vd[v0:v0 + vc, 0:3] += np.random.default_rng(2).normal(0, 0.05, (vc, 3)).astype(np.float32)
    assert lib.orc_refit_blas(orc._p(n2), n2.size, orc._p(pool.triIndex), pool.triIndex.size, orc._p(vd), vd.size, r, e)
    f = n2.view(np.float32)
    for i in range(r, e):
        if n2[i, 7] != 0xFFFFFFFF:
            off, cnt = int(n2[i, 7] & 0xFFFFFF), int(n2[i, 7] >> 24)
            P = vd[pool.triIndex[off:off + cnt].reshape(-1), 0:3]
            assert np.array_equal(f[i, 0:3], P.min(0)) and np.array_equal(f[i, 3:6], P.max(0))
        else:
            l, rr = i + 1, int(n2[i + 1, 6])
            assert np.array_equal(f[i, 0:3], np.minimum(f[l, 0:3], f[rr, 0:3]))
    # layout violation: right child outside (left, end) -> false
    bad = n2.copy()
    first_interior = next(i for i in range(r, e) if bad[i, 7] == 0xFFFFFFFF)
    bad[first_interior + 1, 6] = e + 3
    assert lib.orc_refit_blas(orc._p(bad), bad.size, orc._p(pool.triIndex), pool.triIndex.size, orc._p(vd), vd.size,
                              r, e) == 0


def test_bvh_closest_matches_brute_force(orc, room):
    s, pool, mats, order, live, aabb = room
    lib = orc.load()
    keep = []
    S = orc.scene_struct(pool, mats, keep=keep)
    rng = np.random.default_rng(5)
    n = 3000
    ro = rng.uniform(0.3, 9.7, (n, 3)).astype(np.float32)
    rd = rng.normal(size=(n, 3))
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    t1, t2 = np.zeros(n), np.zeros(n)
    a1, a2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    i1, i2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib.orc_closest(C.byref(S), orc._p(ro), orc._p(rd), n, 0, 0, orc._p(t1), orc._p(a1), orc._p(i1), None, orc.threads())
    lib.orc_closest(C.byref(S), orc._p(ro), orc._p(rd), n, 0, 1, orc._p(t2), orc._p(a2), orc._p(i2), None, orc.threads())
    assert (a1 >= 0).mean() > 0.99  # a closed room: nearly every ray hits
    same = (a1 == a2) & (i1 == i2)
    tie = np.abs(t1 - t2) <= 1e-12 * np.maximum(1, np.abs(t1))
    assert (same | tie).all()
    assert np.allclose(t1, t2, rtol=1e-12)


def test_any_hit_agrees_with_closest(orc, room):
    s, pool, mats, order, live, aabb = room
    lib = orc.load()
    keep = []
    S = orc.scene_struct(pool, mats, keep=keep)
    rng = np.random.default_rng(6)
    n = 2000
    ro = rng.uniform(0.3, 9.7, (n, 3)).astype(np.float32)
    rd = rng.normal(size=(n, 3))
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    md = rng.uniform(0.1, 6.0, n).astype(np.float32)
    t = np.zeros(n)
    tri, inst = np.zeros(n, np.int32), np.zeros(n, np.int32)
    blk = np.zeros(n, np.uint8)
    lib.orc_closest(C.byref(S), orc._p(ro), orc._p(rd), n, 0, 0, orc._p(t), orc._p(tri), orc._p(inst), None, orc.threads())
    lib.orc_any(C.byref(S), orc._p(ro), orc._p(rd), orc._p(md), n, orc._p(blk), orc.threads())
    expect = (tri >= 0) & (t < md)
    assert np.array_equal(blk.astype(bool), expect)
