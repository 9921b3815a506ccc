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


# ------------------------------------------------------- combined receiver
def _const_atlas(shape_hw, rgba):
    a = np.zeros(shape_hw + (4,), np.float16)
    a[...] = np.asarray(rgba, np.float16)
    return a.view(np.uint16).copy()


def _rdirs(n, seed, rough=(0.0, 1.0)):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    out = np.zeros((n, 4), np.float32)
    out[:, :3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    out[:, 3] = rng.uniform(rough[0], rough[1], n)
    return out


def test_combined_receiver_irradiance_is_the_plain_gather_and_zero_intensity_has_no_layer():
    g = _grid()
    G = orc.grid_struct(g)
    a = _random_atlas(g, 11)
    d = _random_atlas(g, 12)
    r = g["res"]
    rough = _const_atlas((r[1] * r[2] * 8, r[0] * 8), (0.5, 0.6, 0.7, 0.8))
    pos, nv = _points(300, 13)
    rd = _rdirs(300, 14)
    for prm in (orc.gather_params(), orc.gather_params(chebyStrength=1.0, chebyBias0=0.02)):
        plain, _ = orc.gather(G, a, d, prm, pos, nv, nv)
        irr, refl, _ = orc.gather_combined(G, a, d, orc.reflect_atlas(rough), prm, pos, nv, nv, rd)
        assert np.allclose(irr, plain, rtol=1e-12, atol=1e-15)
        assert (refl[:, 3] > 0).all()
    p0 = orc.gather_params(reflectionIntensity=0.0)
    _, refl, _ = orc.gather_combined(G, a, d, orc.reflect_atlas(rough), p0, pos, nv, nv, rd)
    assert np.abs(refl).max() == 0.0


def test_combined_receiver_constant_lobes_resolve_to_their_values():
    """Normalised tap weights: a constant rough atlas gives its value times the
    reflection weight; with a glossy atlas the two blend by smoothstep(0.22,
    0.58, roughness); receivers rougher than the limit get no layer."""
    g = _grid()
    G = orc.grid_struct(g)
    a = _random_atlas(g, 21)
    d = _random_atlas(g, 22)
    r = g["res"]
    P = r[0] * r[1] * r[2]
    rough_v, glossy_v = np.array([0.5, 0.25, 0.75, 0.5]), np.array([1.5, 1.0, 0.5, 1.0])
    rough = _const_atlas((r[1] * r[2] * 8, r[0] * 8), rough_v)
    tx = int(np.ceil(np.sqrt(P)))
    ty = -(-P // tx)
    glossy = _const_atlas((ty * 10, tx * 10), glossy_v)
    pos, nv = _points(400, 23)
    rd = _rdirs(400, 24)
    prm = orc.gather_params(reflectionIntensity=0.75, roughnessLimit=0.9)
    _, refl, near = orc.gather_combined(G, a, d, orc.reflect_atlas(rough), prm, pos, nv, nv, rd)
    rw = np.where(rd[:, 3] <= np.float32(0.9), 0.75, 0.0)[:, None]
    assert np.allclose(refl, rough_v[None, :] * rw, rtol=1e-12, atol=1e-15)
    _, refl, _ = orc.gather_combined(G, a, d, orc.reflect_atlas(rough, glossy, 8, tx), prm, pos, nv, nv, rd)
    t = np.clip((rd[:, 3].astype(np.float64) - 0.22) / (0.58 - 0.22), 0, 1)
    m = (t * t * (3 - 2 * t))[:, None]
    want = (glossy_v[None, :] * (1 - m) + rough_v[None, :] * m) * rw
    assert np.allclose(refl, want, rtol=1e-12, atol=1e-15)
