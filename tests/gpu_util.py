"""Shared set-up for the GPU parity tests: one scene on the CUDA path and the
same scene, grid, lights and parameters on the oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np

from speedball_b200 import _abi
from speedball_b200.field import ProbeField

import orc

# Parity tolerances of the update path: hit t 1e-5 relative, texels
# 1e-3 relative; near-tie exemption when the two nearest candidates are within
# 1e-6 relative.
T_REL = 1e-5
TEXEL_REL = 1e-3
TIE_REL = 1e-6


def grid_dict(g: _abi.sb_grid) -> dict:
    return dict(gridMin=[g.gridMin[a] for a in range(3)], gridSize=[g.gridSize[a] for a in range(3)],
                res=[g.res[a] for a in range(3)], rays=g.raysPerProbe, maxDist=g.maxDist, cellMin=g.cellMin)


def make_field(scene, record=True, rays=None, **opts) -> ProbeField:
    m = scene.meta
    g = m["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1,
                   rays=rays or g["rays"], clusteredLighting=m.get("clustered", False),
                   hysteresis=m.get("hysteresis"), jitterMode=m.get("jitter", "gated"), recordHits=record, **opts)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)  # one solve covers every probe
    return f


def read(field: ProbeField, key: str, count: int, dtype, cascade: int = 0) -> np.ndarray:
    out = np.zeros(count, dtype)
    _abi.check(field._lib.sb_read_buffer(field.ctx, _abi.BUF[key] | (cascade << 8), 0, count, _abi.ptr(out)),
               field.ctx)
    return out


class OracleMirror:
    """The oracle's copy of a field's scene, grid, lights and FP64 state."""

    def __init__(self, field: ProbeField, fp32: bool = False, cascade: int = 0):
        self.field = field
        self.cascade = cascade
        pool = field.pool
        self.pool = pool
        self.materials = read(field, "MATERIALS", pool.materials.shape[0], np.float32)
        self.nodes = read(field, "BVH_NODES", pool.bvhNodes.size, np.uint32).reshape(-1, 8)
        self.vertex = read(field, "VERTEX_DATA", pool.vertexData.size, np.float32).reshape(-1, 8)
        self.keep = []
        self.scene = orc.scene_struct(pool, self.materials, nodes=self.nodes, vertex=self.vertex, keep=self.keep)
        self.gdict = grid_dict(field.cascadeGrid(cascade))
        self.grid = orc.grid_struct(self.gdict)
        self.g0dict = grid_dict(field.grid)
        self.grid0 = orc.grid_struct(self.g0dict)
        sc = field._scene
        from speedball_b200.field import selectGiLightRecords
        g = self.gdict
        g0 = self.g0dict
        recs, analytic, n_emit = selectGiLightRecords(sc.lights, field._clustered, g0["gridMin"],
                                                      [g0["gridMin"][a] + g0["gridSize"][a] for a in range(3)])
        self.emitters = (analytic, n_emit)
        self.light_count = recs.shape[0]
        self.clustered = field._clustered
        self.arena = orc.light_arena(recs, self.clustered, g0)
        self.fp32 = fp32
        self.irr, self.depth, self.atlas, self.depth_atlas = orc.new_state(g, fp32)
        r = g["res"]
        self.evis = np.zeros(r[0] * r[1] * r[2] * 16, np.float32 if fp32 else np.float64)
        tier = _abi.REFLECT_TIERS[field.getReflectionQuality()]
        self.rf = orc.ReflectState(g, tier, fp32) if tier else None

    def reflect_state(self):
        rf = self.rf
        if rf is None:
            return None
        return (rf.rough.copy(), rf.rough_atlas.copy(), rf.glossy_num.copy(), rf.glossy_den.copy(),
                rf.glossy_atlas.copy(), rf.phase)

    def restore_reflect(self, st):
        if st is None:
            return
        rf = self.rf
        rf.rough[...], rf.rough_atlas[...], rf.glossy_num[...], rf.glossy_den[...], rf.glossy_atlas[...] = st[:5]
        rf.phase = st[5]

    def params(self) -> np.ndarray:
        return self.field._params.to_array()

    def solve(self, offset: int, updated: int, replay: dict | None = None, want: bool = True,
              params: np.ndarray | None = None, evis_replay: np.ndarray | None = None):
        n = updated * self.gdict["rays"]
        io = orc.OrcSolveIO()
        self.evis_samples = None
        if self.emitters[1]:
            io.emitterVis = orc._p(self.evis)
            self.evis_samples = np.zeros(updated * 16, self.evis.dtype)
            io.emitterSampleOut = orc._p(self.evis_samples)
            if evis_replay is not None:
                self._evis_replay = np.ascontiguousarray(evis_replay, self.evis.dtype)
                io.emitterVisReplay = orc._p(self._evis_replay)
        out = {}
        if want:
            out = dict(rays=np.zeros(n * 4, np.float32 if self.fp32 else np.float64), tri=np.zeros(n, np.int32),
                       inst=np.zeros(n, np.int32), second=np.zeros(n, np.float32 if self.fp32 else np.float64),
                       tested=np.zeros(n, np.uint64), blocked=np.zeros(n, np.uint64))
            io.rayOut = orc._p(out["rays"]); io.hitTri = orc._p(out["tri"]); io.hitInst = orc._p(out["inst"])
            io.secondT = orc._p(out["second"]); io.tested = orc._p(out["tested"]); io.blocked = orc._p(out["blocked"])
        if replay is not None:
            io.replayTri = orc._p(replay["tri"]); io.replayInst = orc._p(replay["inst_word"])
            io.replayBlocked = orc._p(replay["blocked"])
        if self.rf is not None:
            self.rf.attach(io)
        orc.solve(self.scene, self.arena, self.light_count, self.clustered, self.grid, self.grid0,
                  self.params() if params is None else params,
                  offset, updated, self.irr, self.depth, self.atlas, self.depth_atlas, fp32=self.fp32, io=io, emitters=self.emitters)
        if self.rf is not None:
            self.rf.advance()
        return out


def gpu_records(field: ProbeField, n: int, cascade: int = 0) -> dict:
    hits = read(field, "HIT_RECORDS", n * 4, np.uint32, cascade).reshape(n, 4)
    vis = read(field, "VISIBILITY", n * 4, np.uint32, cascade).reshape(n, 4)
    tri = hits[:, 0].view(np.int32).copy()
    word = hits[:, 1].copy()
    inst = np.where(tri >= 0, word & 0x7FFFFFFF, 0xFFFFFFFF).astype(np.uint32).view(np.int32)
    t = hits[:, 2].view(np.float32).copy()
    tested = vis[:, 0].astype(np.uint64) | (vis[:, 1].astype(np.uint64) << np.uint64(32))
    unblocked = vis[:, 2].astype(np.uint64) | (vis[:, 3].astype(np.uint64) << np.uint64(32))
    blocked = tested & ~unblocked
    # replay input keeps the facing bit in bit 31 of the instance word
    return dict(tri=np.ascontiguousarray(tri), inst=np.ascontiguousarray(inst),
                inst_word=np.ascontiguousarray(word.view(np.int32)), facing=(word >> 31).astype(bool), t=t,
                blocked=np.ascontiguousarray(blocked))


def half_to_f(a: np.ndarray) -> np.ndarray:
    return a.view(np.float16).astype(np.float64)


def texel_rel_err(g: np.ndarray, o: np.ndarray) -> np.ndarray:
    """|g - o| / max(|o|, floor): relative error with an absolute floor of 1e-3
    of the largest magnitude for near-black texels."""
    floor = max(1e-3 * float(np.abs(o).max()), 1e-12)
    return np.abs(g - o) / np.maximum(np.abs(o), floor)


def check_hits(scene: orc.OrcScene, ro: np.ndarray, rd: np.ndarray, g_tri, g_inst, g_t, o_tri, o_inst, o_t,
               g_ro: np.ndarray | None = None, g_rd: np.ndarray | None = None) -> dict:
    """Hit-ID parity at the near-tie bar: every ray whose GPU closest hit
    differs from the FP64 oracle's on ray (ro, rd) must be explained, ray by
    ray, by the oracle (orc.explain_hits: a near-tie within 1e-6 relative, an
    edge graze within the FP32 rounding bound of that triangle's barycentric
    test, or a t order within the FP32 bound of the two t); no share of rays is
    waived. Hit t: the GPU's t is within 1e-5 relative of the FP64 t of the
    pair it reports, on the ray it traced ((g_ro, g_rd), the FP32 ray, when
    given; else (ro, rd)). Returns the count of rays per code, and the largest
    relative t difference against the FP64 ray as well."""
    code, gt = orc.explain_hits(scene, ro, rd, g_tri, g_inst, o_tri, o_inst, o_t)
    counts = {orc.HIT_CODES[k]: int(v) for k, v in enumerate(np.bincount(code, minlength=6))}
    bad = np.flatnonzero(code == 5)
    assert bad.size == 0, (counts, [(int(i), int(g_tri[i]), int(o_tri[i]), float(g_t[i]), float(o_t[i]), float(gt[i]))
                                    for i in bad[:6]])
    g_hit = np.asarray(g_tri) >= 0
    g_t = np.asarray(g_t, np.float64)
    if g_ro is not None:
        tt = orc.pair_t(scene, g_ro.astype(np.float64), g_rd.astype(np.float64), g_tri, g_inst)
    else:
        tt = orc.pair_t(scene, ro, rd, g_tri, g_inst)
    ok = g_hit & (tt > 0)
    assert ok.sum() == g_hit.sum(), (int(g_hit.sum()), int(ok.sum()))
    rel = np.abs(g_t[ok] - tt[ok]) / tt[ok]
    counts["t_rel_max"] = float(rel.max()) if rel.size else 0.0
    assert counts["t_rel_max"] <= T_REL, counts["t_rel_max"]
    if g_ro is not None:
        # the FP32 ray against the FP64 one, and what that rounding does to t
        t64 = orc.pair_t(scene, ro, rd, g_tri, g_inst)
        both = ok & (t64 > 0)
        counts["t_rel_max_vs_fp64_ray"] = float((np.abs(g_t[both] - t64[both]) / t64[both]).max()) if both.any() else 0.0
        counts["t_rel_gt_1e-5_vs_fp64_ray"] = int((np.abs(g_t[both] - t64[both]) > T_REL * t64[both]).sum())
        dang = np.linalg.norm(g_rd.astype(np.float64) / np.linalg.norm(g_rd.astype(np.float64), axis=1, keepdims=True)
                              - rd, axis=1)
        counts["ray_dir_err_max_rad"] = float(dang.max())
        assert dang.max() <= 4e-7, dang.max()
        # FP32 probe origins: a few roundings at the scale of the grid's coordinates
        dorg = np.abs(g_ro.astype(np.float64) - ro).max(axis=1) / max(float(np.abs(ro).max()), 1.0)
        counts["ray_origin_rel_err_max"] = float(dorg.max())
        assert dorg.max() <= 4e-7, dorg.max()
    return counts


class SceneTail:
    """The oracle's own per-frame scene state for motion: the deforming mesh's
    vertices and BLAS refit (updateDeforms, spectral_scene.js:1831-1927 with
    refitFlatBlasRange), the moved instances' rows and the TLAS refit of the
    partition frozen at the build (updateTransforms, 1402-1514). It writes into
    an OracleMirror's arrays in place and checks them bit for bit against the
    GPU's copies."""

    def __init__(self, mirror: OracleMirror):
        self.m = mirror
        pool = mirror.pool
        mats0, order0, live0, aabb0 = orc.compute_tail(pool, nodes=mirror.nodes)
        self.order = order0
        self.tl = np.ascontiguousarray(mats0[pool.tlasBase:].copy())
        self.world = pool.inst_world.copy()
        n = pool.instCount
        self.inv = np.zeros((n, 12), np.float32)
        self.det = np.zeros(n, np.float32)
        self.aabb = np.zeros((n, 9))

    def apply(self, deformed: dict, moved: dict):
        """deformed: mesh -> (V,3) float32 positions; moved: instance -> 4x4 world."""
        lib = orc.load()
        m, pool = self.m, self.m.pool
        for mesh, pos in deformed.items():
            vb, vc = int(pool.vert_base[mesh]), int(pool.vert_count[mesh])
            m.vertex[vb:vb + vc, 0:3] = pos
            assert lib.orc_refit_blas(orc._p(m.nodes), m.nodes.size, orc._p(pool.triIndex), pool.triIndex.size,
                                      orc._p(m.vertex), m.vertex.size, int(pool.blas_root[mesh]),
                                      int(pool.blas_end[mesh])) == 1
        for i, w in moved.items():
            self.world[i] = np.asarray(w, np.float64).T.reshape(16)
        lb = np.ascontiguousarray(orc.local_bounds(m.nodes, pool.inst_root))
        lib.orc_compute_instances(orc._p(self.world), orc._p(pool.inst_active), orc._p(lb), pool.instCount,
                                  orc._p(self.inv), orc._p(self.det), orc._p(self.aabb))
        ib = pool.instBase
        for slot, src in enumerate(self.order):
            m.materials[ib + slot * 28: ib + slot * 28 + 12] = self.inv[src]
            m.materials[ib + slot * 28 + 14] = self.det[src]
        live = np.ascontiguousarray(self.aabb[self.order, 0:6].astype(np.float32))
        assert lib.orc_refit_tlas_range(orc._p(self.tl), self.tl.size, orc._p(live), live.size, 0,
                                        pool.tlasNodeCount)
        m.materials[pool.tlasBase:] = self.tl

    def check_gpu(self):
        f, m = self.m.field, self.m
        for key, arr in (("BVH_NODES", m.nodes), ("VERTEX_DATA", m.vertex), ("MATERIALS", m.materials)):
            got = read(f, key, arr.size, arr.dtype).reshape(arr.shape)
            assert np.array_equal(got.view(np.uint32), arr.view(np.uint32)), key


def gpu_probe_rays(f: ProbeField, offset: int, updated: int, cascade: int = 0):
    """The FP32 probe rays the GPU traced for a solve (sb_probe_rays)."""
    n = updated * f.getRays()
    ro = np.zeros((n, 3), np.float32)
    rd = np.zeros((n, 3), np.float32)
    _abi.check(f._lib.sb_probe_rays(f.ctx, cascade, offset, updated, _abi.ptr(ro), _abi.ptr(rd)), f.ctx)
    return ro, rd


def solve_parity(f: ProbeField, mirror: OracleMirror, frame: dict, sched_params: np.ndarray) -> dict:
    """After the GPU tick `frame`: independent FP64 solve (hit IDs and t of every
    ray of the solve), then the oracle's replay of the GPU's hit and shadow
    decisions advances its state; irradiance and depth atlases within 1e-3."""
    off, upd = frame["probeOffset"], frame["updatedCount"]
    ci = mirror.cascade
    n = upd * f.getRays()
    rec = gpu_records(f, n, ci)
    saved = (mirror.irr.copy(), mirror.depth.copy(), mirror.atlas.copy(), mirror.depth_atlas.copy(),
             mirror.evis.copy())
    saved_rf = mirror.reflect_state()
    ind = mirror.solve(off, upd, replay=None, params=sched_params)
    samples = mirror.evis_samples
    mirror.irr, mirror.depth, mirror.atlas, mirror.depth_atlas, evis_before = saved
    mirror.evis[...] = evis_before
    mirror.restore_reflect(saved_rf)
    gpu_evis = None
    if mirror.emitters[1]:
        # the GPU's visibility history after this solve, and the samples it implies
        # (after = 0.2 sample + 0.8 before, gi_probes.js:2258-2259)
        gpu_evis = read(f, "EMITTER_VIS", mirror.evis.size, np.float32, ci).astype(np.float64)
        probes = (off + np.arange(upd)) % (mirror.evis.size // 16)
        ne = mirror.emitters[1]
        before = evis_before.reshape(-1, 16)[probes, :ne]
        after = gpu_evis.reshape(-1, 16)[probes, :ne]
        g_samp = np.rint((after - np.float32(0.8) * before) / np.float32(0.2))
        o_samp = samples.reshape(upd, 16)[:, :ne]
        emitter_agree = (g_samp == o_samp).mean(axis=0)
    ro, rd = orc.probe_rays(mirror.grid, sched_params[0], off, upd)
    g_ro, g_rd = gpu_probe_rays(f, off, upd, ci)
    counts = check_hits(mirror.scene, ro, rd, rec["tri"], rec["inst"], rec["t"], ind["tri"], ind["inst"],
                        ind["rays"][3::4], g_ro, g_rd)
    mirror.solve(off, upd, replay=rec, params=sched_params, evis_replay=gpu_evis)
    ga = half_to_f(read(f, "IRRADIANCE_ATLAS", mirror.atlas.size, np.uint16, ci))
    oa = half_to_f(mirror.atlas.reshape(-1))
    err = texel_rel_err(ga, oa)
    gd = half_to_f(read(f, "DEPTH_ATLAS", mirror.depth_atlas.size, np.uint16, ci))
    od = half_to_f(mirror.depth_atlas.reshape(-1))
    derr = texel_rel_err(gd, od)
    assert err.max() <= TEXEL_REL, (err.max(), int((err > TEXEL_REL).sum()))
    assert derr.max() <= TEXEL_REL, (derr.max(), int((derr > TEXEL_REL).sum()))
    counts.update(irr_err=float(err.max()), depth_err=float(derr.max()), lit=float(np.abs(oa).max()),
                  hit_share=float((rec["tri"] >= 0).mean()))
    if gpu_evis is not None:
        counts["emitter_sample_agreement"] = [float(x) for x in emitter_agree]
    if mirror.rf is not None:
        counts.update(reflection_parity(f, mirror))
    return counts


def reflection_parity(f: ProbeField, mirror: OracleMirror) -> dict:
    """The reflection lobes after a replayed solve: the rough history and atlas
    and (tiers high / ultra) the glossy numerator, support and atlas, each
    within 1e-3 relative of the oracle's (colour and coverage separately, floor
    1e-3 of the largest magnitude)."""
    rf, ci = mirror.rf, mirror.cascade
    out = {}

    def cmp(name, g, o, stride):
        g = g.reshape(-1, stride)
        o = o.reshape(-1, stride)
        errs = [texel_rel_err(g[:, :3], o[:, :3]).max()] + ([texel_rel_err(g[:, 3], o[:, 3]).max()] if stride == 4 else [])
        e = float(max(errs))
        assert e <= TEXEL_REL, (name, e)
        out[name] = e

    cmp("rough_hist_err", read(f, "ROUGH_SPECULAR", rf.rough.size, np.float32, ci), rf.rough, 4)
    cmp("rough_atlas_err", half_to_f(read(f, "ROUGH_ATLAS", rf.rough_atlas.size, np.uint16, ci)),
        half_to_f(rf.rough_atlas.reshape(-1)), 4)
    out["rough_coverage_mean"] = float(rf.rough.reshape(-1, 4)[:, 3].mean())
    if rf.tier >= 2:
        gd = read(f, "GLOSSY_WEIGHT", rf.glossy_den.size, np.float32, ci)
        err = texel_rel_err(gd, rf.glossy_den)
        assert err.max() <= TEXEL_REL, ("glossy_den", float(err.max()))
        out["glossy_den_err"] = float(err.max())
        cmp("glossy_num_err", read(f, "GLOSSY_SPECULAR", rf.glossy_num.size, np.float32, ci), rf.glossy_num, 4)
        cmp("glossy_atlas_err", half_to_f(read(f, "GLOSSY_ATLAS", rf.glossy_atlas.size, np.uint16, ci)),
            half_to_f(rf.glossy_atlas.reshape(-1)), 4)
        lay = f.reflectionLayout(ci)
        assert lay["glossyPhase"] == rf.phase, (lay, rf.phase)
    return out
