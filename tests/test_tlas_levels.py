"""The GPU TLAS build runs level by level (every interior segment of a level
sorted at once, finished leaves frozen in place); this checks that schedule
against the oracle's recursive buildTlasRecords (spectral_scene.js:973-1003)
on scenes of 65, 30 and 400 instances (CPU only)."""
import numpy as np
import pytest

from speedball_b200 import scene as sc
from speedball_b200 import synth


def level_sync_order(aabb):
    n = aabb.shape[0]

    def nodes(m):
        return 1 if m <= 2 else 1 + nodes(m >> 1) + nodes(m - (m >> 1))

    order = list(range(n))
    segs = [(0, n, 0)]
    while segs:
        seg_of = [None] * n
        axis = {}
        for si, (lo, hi, idx) in enumerate(segs):
            for j in range(lo, hi):
                seg_of[j] = si
            members = [order[j] for j in range(lo, hi)]
            mn, mx = aabb[members, 0:3].min(0), aabb[members, 3:6].max(0)
            if hi - lo <= 2:
                axis[si] = None
            else:
                ex, ey, ez = mx - mn
                axis[si] = 0 if (ex >= ey and ex >= ez) else (1 if ey >= ez else 2)
        recs = []
        for j in range(n):
            si = seg_of[j]
            group = j if si is None else segs[si][0]
            ax = None if si is None else axis[si]
            key = 0.0 if ax is None else float(aabb[order[j], 6 + ax])
            recs.append((group, key, j))
        recs.sort()
        order = [order[r[2]] for r in recs]
        nxt = []
        for lo, hi, idx in segs:
            if hi - lo > 2:
                mid = (lo + hi) >> 1
                nxt += [(lo, mid, idx + 1), (mid, hi, idx + 1 + nodes(mid - lo))]
        segs = nxt
    return np.array(order, np.uint32)


@pytest.mark.parametrize("n", [65, 30, 400])
def test_level_synchronous_build_equals_recursive(orc, n):
    rng = np.random.default_rng(n)
    if n == 65:
        pool = sc.build_pool(synth.room_spheres(0))
        _, order, _, aabb = orc.compute_tail(pool)
    else:
        mn = rng.uniform(-50, 50, (n, 3))
        mn[rng.integers(0, n, n // 5)] = 7.0  # ties on every axis
        mx = mn + rng.uniform(0.0, 5.0, (n, 3))
        aabb = np.concatenate([mn, mx, (mn + mx) * 0.5], 1)
        tl = np.zeros((2 * n + 2, 12), np.float32)
        order = np.zeros(n, np.uint32)
        orc.load().orc_build_tlas(orc._p(np.ascontiguousarray(aabb)), n, orc._p(tl), orc._p(order), None)
    assert np.array_equal(level_sync_order(aabb), order)
