"""CPU checks of the oracle's receiver-gather restatement (orc_gather.hpp)."""
import ctypes as C

import numpy as np

import orc


def _grid():
    return orc.grid_dict([0.0, 0.0, 0.0], [8.0, 6.0, 4.0], [5, 4, 3], 64)


def _random_atlas(g, seed):
    rng = np.random.default_rng(seed)
    r = g["res"]
    W, H = r[0] * 8, r[1] * r[2] * 8
    vals = rng.uniform(0.05, 2.0, (H, W, 4)).astype(np.float16)
    vals[..., 3] = 1.0
    return vals.view(np.uint16).copy()


def _points(n, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform([0.2, 0.2, 0.2], [7.8, 5.8, 3.8], (n, 3))
    nv = rng.normal(size=(n, 3))
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    a = np.zeros((n, 4), np.float32)
    a[:, :3] = nv
    return pos, a


def test_constant_atlas_gathers_its_value():
    g = _grid()
    G = orc.grid_struct(g)
    r = g["res"]
    atlas = np.zeros((r[1] * r[2] * 8, r[0] * 8, 4), np.float16)
    atlas[..., :3] = np.float16(0.625)
    atlas[..., 3] = 1.0
    a = atlas.view(np.uint16).copy()
    pos, nv = _points(500, 1)
    out, _ = orc.gather(G, a, a, orc.gather_params(intensity=2.0), pos, nv, nv)
    assert np.allclose(out, 1.25, rtol=1e-12)


def test_default_gather_is_the_trace_side_atlas_read_at_the_biased_point():
    """With chebyStrength 0 the receiver gather is the trilinear 8-tap read of
    the trace kernel's one-bounce lookup (sampleAtlas, gi_probes.js:1941-1974)
    at P = position + normalBias * N."""
    g = _grid()
    G = orc.grid_struct(g)
    a = _random_atlas(g, 2)
    pos, nv = _points(300, 3)
    bias = 0.04
    out, _ = orc.gather(G, a, a, orc.gather_params(normalBias0=bias), pos, nv, nv)
    lib = orc.load()
    for i in range(pos.shape[0]):
        P = (pos[i, :3].astype(np.float64) + nv[i, :3].astype(np.float64) * np.float64(np.float32(bias)))
        N = nv[i, :3].astype(np.float64)
        v = (C.c_double * 3)()
        lib.orc_sample_atlas(C.byref(G), orc._p(a), orc._p(np.ascontiguousarray(P)), orc._p(np.ascontiguousarray(N)), v)
        assert np.allclose(out[i], v[:], rtol=1e-12, atol=1e-15), i


def test_visible_surfaces_leave_only_the_wrap_weight():
    """Depth moments far beyond every sample (all surfaces visible: dist <= m1)
    leave only the wrap weight acting when visibility is on: the result moves
    away from the plain trilinear one but stays a convex combination of the
    atlas values."""
    g = _grid()
    G = orc.grid_struct(g)
    a = _random_atlas(g, 4)
    r = g["res"]
    far = np.zeros((r[1] * r[2] * 8, r[0] * 8, 4), np.float16)
    far[..., 0] = 50.0
    far[..., 1] = 2500.0
    far[..., 3] = 1.0
    dfar = far.view(np.uint16).copy()
    pos, nv = _points(400, 5)
    plain, _ = orc.gather(G, a, dfar, orc.gather_params(), pos, nv, nv)
    # with visibility on and every surface visible (dist <= m1), only the wrap weight acts
    vis, near = orc.gather(G, a, dfar, orc.gather_params(chebyStrength=1.0), pos, nv, nv)
    assert np.all(np.isfinite(vis)) and np.abs(vis - plain).max() > 1e-3
    # wrap weights are >= 0.05^2 of the trilinear weights: the result stays in the atlas' value range
    assert vis.min() >= 0.0 and vis.max() <= 2.0 + 1e-9
