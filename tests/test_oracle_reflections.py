"""The oracle's reflection lobes (reflectionQuality rough / high / ultra,
gi_probes.js:60-75) against a second, independent numpy restatement. CPU only.

Rays are fed to the oracle's blend directly (OrcSolveIO.rayIn), so every case
is exact and small:
  * rough lobe (power 8, gi_probes.js:2388-2404, 2505-2522): the first solve
    seeds the history with the current lobe (depth unseeded), the second
    blends with the steady retention; local hits count, misses count only with
    the sky fallback, encoded unshaded hits never;
  * the rough atlas is the history with the canonical mirrored gutter, binary16;
  * glossy lobe (power 64, glossyKernel 2538-2686) on 18x18 (ultra) and 10x10
    (high) tiles with mirrored gutters: per-ray-mean numerator and support,
    the interleave of tier high (texels of one parity per solve), the retention
    exponent x interval, the packed glossy atlas;
  * the trace's rough-unshaded encoding (2055-2062): with every material
    metallic, each hit is stored as -(t + 2) and the lobes ignore it.
"""
import math

import numpy as np

import orc
from speedball_b200 import synth

N = 64
RES = (3, 3, 2)
IDX = {n: i for i, n in enumerate(orc.ORC_PARAM_NAMES)}


def _oct_decode(u, v):
    fx, fy = u * 2 - 1, v * 2 - 1
    nz = 1 - abs(fx) - abs(fy)
    t = max(-nz, 0.0)
    nx = fx + (-t if fx >= 0 else t)
    ny = fy + (-t if fy >= 0 else t)
    d = np.array([nx, ny, nz])
    return d / np.linalg.norm(d)


def _ray_dirs(n, jitter=0.0):
    k = np.arange(n, dtype=np.float64)
    u = np.mod((k + 0.5) / n + jitter, 1.0)
    z = 1 - 2 * u
    r = np.sqrt(np.maximum(0.0, 1 - z * z))
    phi = k * math.pi * (3 - math.sqrt(5)) + 2 * math.pi * jitter
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def _mirror(lx, ly, tile, oct_):
    edge, lo, hi = tile - 1, 1, oct_
    onL, onR, onT, onB = lx == 0, lx == edge, ly == 0, ly == edge
    colB, rowB = onL or onR, onT or onB
    if colB and rowB:
        return (hi if onL else lo), (hi if onT else lo)
    if rowB:
        return edge - lx, (lo if onT else hi)
    if colB:
        return (lo if onL else hi), edge - ly
    return lx, ly


class _Setup:
    def __init__(self, tier):
        s = synth.room_spheres(0)
        pool = orc.OrcPool(s)
        mats, _, _, _ = orc.compute_tail(pool)
        self.keep = [pool]
        self.S = orc.scene_struct(pool, mats, keep=self.keep)
        self.g = orc.grid_dict((1.0, 1.0, 1.0), (8.0, 8.0, 8.0), RES, N)
        self.G = orc.grid_struct(self.g)
        recs, _, _ = orc.select_light_records(s.lights, False, self.g["gridMin"], [9.0, 9.0, 9.0])
        self.arena = orc.light_arena(recs, False, None)
        self.nl = recs.shape[0]
        self.prm = orc.default_params(0.97)
        self.irr, self.depth, self.atlas, self.datlas = orc.new_state(self.g)
        self.rf = orc.ReflectState(self.g, tier)
        self.P = RES[0] * RES[1] * RES[2]

    def blend(self, rays, prm=None):
        io = orc.OrcSolveIO()
        rays = np.ascontiguousarray(rays, np.float64)
        io.rayIn = orc._p(rays)
        self.rf.attach(io)
        orc.solve(self.S, self.arena, self.nl, False, self.G, self.G, self.prm if prm is None else prm, 0, self.P,
                  self.irr, self.depth, self.atlas, self.datlas, io=io, nthreads=2)
        self.rf.advance()


def _rays(rng, P, sky_share=0.3, unshaded_share=0.2):
    rays = np.zeros((P, N, 4))
    rays[..., :3] = rng.uniform(0.0, 3.0, (P, N, 3))
    u = rng.uniform(size=(P, N))
    t = rng.uniform(0.5, 9.0, (P, N))
    rays[..., 3] = np.where(u < sky_share, -1.0, np.where(u < sky_share + unshaded_share, -(t + 2.0), t))
    return rays


def _valid(hitT, sky_valid):
    return np.where(hitT >= 0, 1.0, np.where(hitT == -1.0, sky_valid, 0.0))


def _rough_lobe(rays, sky_valid):
    """sCur per (probe, interior texel): (rgb, coverage)."""
    dirs = _ray_dirs(N)
    out = np.zeros((rays.shape[0], 36, 4))
    for lane in range(36):
        td = _oct_decode((lane % 6 + 0.5) / 6, (lane // 6 + 0.5) / 6)
        sw = np.maximum(dirs @ td, 0.0) ** 8
        for p in range(rays.shape[0]):
            v = _valid(rays[p, :, 3], sky_valid)
            den = max(sw.sum(), 1e-4)
            out[p, lane, :3] = (rays[p, :, :3] * (sw * v)[:, None]).sum(0) / den
            out[p, lane, 3] = min(max((sw * v).sum() / den, 0.0), 1.0)
    return out


def _rough_hist(rf, P):
    h = rf.rough.reshape(P, 8, 8, 4)
    return np.stack([h[:, lane // 6 + 1, lane % 6 + 1] for lane in range(36)], 1)


def test_rough_lobe_first_and_second_solve():
    su = _Setup(1)
    rng = np.random.default_rng(1)
    r1 = _rays(rng, su.P)
    su.blend(r1.reshape(-1))
    want1 = _rough_lobe(r1, 0.0)  # no sky fallback by default
    got1 = _rough_hist(su.rf, su.P)
    assert np.abs(got1 - want1).max() < 1e-12
    assert (want1[..., 3] > 0).all() and (want1[..., 3] < 1).all()  # a mix of counted and ignored rays
    # second solve: depth is seeded now, the steady retention applies
    r2 = _rays(rng, su.P)
    su.blend(r2.reshape(-1))
    h = su.prm[IDX["hysteresis"]]  # the uniform as stored (float32)
    steady = min(max(h + (1 - h) * 0.25, 1e-6), 1.0) ** 1.0
    want2 = _rough_lobe(r2, 0.0) * (1 - steady) + want1 * steady
    assert np.abs(_rough_hist(su.rf, su.P) - want2).max() < 1e-12


def test_sky_fallback_counts_misses():
    su = _Setup(1)
    prm = su.prm.copy()
    prm[IDX["reflectionSkyFallback"]] = 1.0
    prm[IDX["skyConfigured"]] = 1.0
    rays = np.zeros((su.P, N, 4))
    rays[..., :3] = 0.5
    rays[..., 3] = -1.0  # every ray misses
    su.blend(rays.reshape(-1), prm)
    got = _rough_hist(su.rf, su.P)
    assert np.allclose(got[..., :3], 0.5, atol=1e-12) and np.allclose(got[..., 3], 1.0, atol=1e-12)
    su2 = _Setup(1)
    su2.blend(rays.reshape(-1))  # fallback off: misses are not reflection samples
    got2 = _rough_hist(su2.rf, su2.P)
    assert np.abs(got2).max() == 0.0


def test_rough_atlas_is_the_history_with_the_mirrored_gutter():
    su = _Setup(1)
    rays = _rays(np.random.default_rng(2), su.P)
    su.blend(rays.reshape(-1))
    hist = su.rf.rough.reshape(su.P, 8, 8, 4)
    W = RES[0] * 8
    lib = orc.load()
    for p in range(su.P):
        col = p % RES[0]
        row = (p // (RES[0] * RES[1])) * RES[1] + (p // RES[0]) % RES[1]
        for ly in range(8):
            for lx in range(8):
                sx, sy = _mirror(lx, ly, 8, 6)
                tex = su.rf.rough_atlas.reshape(-1, W, 4)[row * 8 + ly, col * 8 + lx]
                want = [lib.orc_to_half(float(x)) for x in hist[p, sy, sx]]
                assert list(tex) == want


def _glossy_lobe(rays, tile, oct_, sky_valid):
    dirs = _ray_dirs(N)
    P = rays.shape[0]
    num = np.zeros((P, tile * tile, 4))
    den = np.zeros((P, tile * tile))
    for local in range(tile * tile):
        sx, sy = _mirror(local % tile, local // tile, tile, oct_)
        td = _oct_decode((sx - 1 + 0.5) / oct_, (sy - 1 + 0.5) / oct_)
        gw = np.maximum(dirs @ td, 0.0) ** 64
        for p in range(P):
            v = _valid(rays[p, :, 3], sky_valid)
            num[p, local, :3] = (rays[p, :, :3] * (gw * v)[:, None]).sum(0)
            num[p, local, 3] = (gw * v).sum()
            den[p, local] = gw.sum()
    inv = float(np.float32(1.0 / N))
    return num * inv, den * inv


def test_glossy_ultra_numerator_support_and_atlas():
    su = _Setup(3)
    rf = su.rf
    assert (rf.tile, rf.interval, rf.tiles_x, rf.tiles_y) == (18, 1, 5, 4)
    rays = _rays(np.random.default_rng(3), su.P)
    su.blend(rays.reshape(-1))
    num, den = _glossy_lobe(rays, 18, 16, 0.0)
    den = np.maximum(den, 1e-6)  # first solve: empty history, weight 0
    assert np.abs(rf.glossy_num.reshape(su.P, -1, 4) - num).max() < 1e-12
    assert np.abs(rf.glossy_den.reshape(su.P, -1) - den).max() < 1e-13
    lib = orc.load()
    A = rf.glossy_atlas
    for p in (0, 7, su.P - 1):
        col, row = p % rf.tiles_x, p // rf.tiles_x
        for local in range(0, 18 * 18, 37):
            lx, ly = local % 18, local // 18
            n, d = num[p, local], den[p, local]
            want = [lib.orc_to_half(float(n[c] / d)) for c in range(3)] + \
                   [lib.orc_to_half(float(min(max(n[3] / d, 0.0), 1.0)))]
            assert list(A[row * 18 + ly, col * 18 + lx]) == want


def test_glossy_high_interleaves_texel_phases():
    su = _Setup(2)
    rf = su.rf
    assert (rf.tile, rf.interval) == (10, 2)
    rng = np.random.default_rng(4)
    r1 = _rays(rng, su.P, sky_share=0.0, unshaded_share=0.0)
    su.blend(r1.reshape(-1))  # phase 0: even texels only
    d1 = rf.glossy_den.reshape(su.P, 100).copy()
    n1, s1 = _glossy_lobe(r1, 10, 8, 0.0)
    even = np.arange(100) % 2 == 0
    assert (d1[:, ~even] == 0).all()
    assert np.abs(d1[:, even] - np.maximum(s1[:, even], 1e-6)).max() < 1e-13
    r2 = _rays(rng, su.P, sky_share=0.0, unshaded_share=0.0)
    su.blend(r2.reshape(-1))  # phase 1: odd texels, seeded from empty
    d2 = rf.glossy_den.reshape(su.P, 100)
    n2, s2 = _glossy_lobe(r2, 10, 8, 0.0)
    assert np.array_equal(d2[:, even], d1[:, even])
    assert np.abs(d2[:, ~even] - np.maximum(s2[:, ~even], 1e-6)).max() < 1e-13
    r3 = _rays(rng, su.P, sky_share=0.0, unshaded_share=0.0)
    su.blend(r3.reshape(-1))  # phase 0 again: retention ^ (exponent x interval)
    n3, s3 = _glossy_lobe(r3, 10, 8, 0.0)
    h = su.prm[IDX["hysteresis"]]
    gh = min(max(h + (1 - h) * 0.25, 1e-6), 1.0) ** 2.0
    want = np.maximum(s3[:, even] * (1 - gh) + np.maximum(s1[:, even], 1e-6) * gh, 1e-6)
    assert np.abs(rf.glossy_den.reshape(su.P, 100)[:, even] - want).max() < 1e-13
    want_num = n3[:, even] * (1 - gh) + n1[:, even] * gh
    assert np.abs(rf.glossy_num.reshape(su.P, 100, 4)[:, even] - want_num).max() < 1e-12


def test_trace_encodes_unshaded_hits():
    """The room with every material fully metallic: tier rough stores each hit
    as -(t + 2) with the same radiance; the rough lobe then has no samples."""
    s = synth.room_spheres(0)
    s.materials = s.materials.copy()
    s.materials[:, 4] = 1.0  # metalness
    s.materials[:, 7:10] = 0.0  # no emission
    pool = orc.OrcPool(s)
    mats, _, _, _ = orc.compute_tail(pool)
    keep = [pool]
    S = orc.scene_struct(pool, mats, keep=keep)
    g = orc.grid_dict((1.0, 1.0, 1.0), (8.0, 8.0, 8.0), (2, 2, 2), N)
    G = orc.grid_struct(g)
    recs, _, _ = orc.select_light_records(s.lights, False, g["gridMin"], [9.0, 9.0, 9.0])
    arena = orc.light_arena(recs, False, None)
    prm = orc.default_params(0.97)
    out = {}
    for tier in (0, 1):
        irr, depth, atlas, datlas = orc.new_state(g)
        rays = np.zeros(8 * N * 4)
        io = orc.OrcSolveIO()
        io.rayOut = orc._p(rays)
        rf = orc.ReflectState(g, tier) if tier else None
        if rf:
            rf.attach(io)
        orc.solve(S, arena, recs.shape[0], False, G, G, prm, 0, 8, irr, depth, atlas, datlas, io=io, nthreads=2)
        out[tier] = (rays.reshape(-1, 4), depth.copy(), rf)
    r0, r1 = out[0][0], out[1][0]
    hit = r0[:, 3] >= 0
    assert hit.all()  # a closed room
    assert np.array_equal(r1[:, 3], -(r0[:, 3] + 2.0))
    assert np.array_equal(r1[:, :3], r0[:, :3])
    # the blend decodes the depth: (t + 2) - 2 is t up to one rounding
    assert np.allclose(out[0][1], out[1][1], rtol=1e-14, atol=0.0)
    assert np.abs(out[1][2].rough).max() == 0.0
