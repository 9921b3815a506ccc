#!/usr/bin/env python3
"""Benchmark: the full DDGI probe update on the Sponza-scale atrium.

Workload (one "step" = one full update of every probe): the seeded
262,267-triangle atrium (30 meshes, 25 materials, 1 directional + 32 clustered
point lights), 16^3 = 4,096 probes x 64 rays = 262,144 primary rays, with the
per-frame motion lanes: 1 deforming mesh (sinusoidal 2 cm vertex offset: BLAS
refit) and 3 rigidly moving meshes (instance rows + TLAS refit).

  value  probe Mrays/s (primary rays / device time of a step: refit -> TLAS
         refit -> trace + shade -> blend + upload), inputs resident in HBM;
         L2 flushed (256 MiB write) before every timed step.
  e2e    the same metric through the public facade (markDeformsDirty,
         markTransformsDirty, update, atlas read-back) with the step's vertex
         and matrix uploads from page-locked host memory and both RGBA16F
         atlases read back, wall-clock per step.

`--impl reference` times the reference algorithm's CPU implementation (the
FP32 CPU restatement of the path, all host threads) on the same workload.
With --gpus N > 1 (torchrun), every rank runs an independent replica.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "probe Mrays/s (full DDGI update)"
UNIT = "Mrays/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["atrium", "adjoint", "batch", "large", "gather", "build"],
                    default="atrium",
                    help="atrium: the plain probe update (headline); adjoint: one gradient evaluation of the "
                         "differentiated update (64 materials, 32 point lights, 2 feedback solves); batch: 3 "
                         "nested cascades of the atrium + 8 independent atria per frame, batched vs plain; "
                         "large: 2.1M unique / 12.8M instanced triangles, C0 32^3 probes + fitted fine cascade C1, 256 rays, "
                         "binary vs 8-wide scene BVH vs the reference two-level walk")
    ap.add_argument("--reflection", choices=["off", "rough", "high", "ultra"], default="off",
                    help="atrium: the reflection tier of the probe field (both arms); gather: off times "
                         "sb_gather_irradiance, a tier the combined receiver sb_gather_reflections on that tier's "
                         "atlases")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-aux", action="store_true",
                    help="atrium only: skip the batched-form and adjoint measurements added to the line")
    return ap.parse_args()


# --------------------------------------------------------------- distributed
class Dist:
    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ workload
def make_workload():
    from speedball_b200 import synth
    scene = synth.atrium(1)
    return scene


def field_for(scene, device, reflection="off"):
    from speedball_b200.field import ProbeField
    g = scene.meta["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1, rays=g["rays"],
                   clusteredLighting=True, hysteresis=scene.meta["hysteresis"], jitterMode="gated", device=device,
                   reflectionQuality=reflection)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)  # one solve updates all 4,096 probes
    return f


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("SB_CLOCKS_CSV", "/tmp/sb_clocks_%d.csv" % os.getpid()))

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait for its first sample so the
        # samples cover the timed region rather than the time after it
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if self.path.stat().st_size > 0:
                break
            time.sleep(0.01)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cudart():
    from cuda import cudart as rt  # cuda-python: streams, events, L2 flush buffer
    return rt


def ck(res):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError(f"CUDA runtime error {err}")
    return res[1] if isinstance(res, tuple) and len(res) > 1 else None


# --------------------------------------------------------------- our arm
def run_ours(args, dist: Dist):
    from speedball_b200 import _abi
    from speedball_b200 import synth
    from speedball_b200.scene import column_major

    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    scene = make_workload()
    f = field_for(scene, device, args.reflection)
    lib, ctx, pool = f._lib, f.ctx, f.pool
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    _abi.check(lib.sb_set_stream(ctx, C.c_void_p(int(stream))), ctx)
    flush = ck(rt.cudaMalloc(L2_FLUSH_BYTES))
    P = f._probeTotal
    rays = P * f.getRays()
    dm = scene.meta["deformer"]
    movers = scene.meta["movers"]
    root, end = int(pool.blas_root[dm]), int(pool.blas_end[dm])
    W, K = args.warmup, args.steps
    e0 = ck(rt.cudaEventCreate())
    e1 = ck(rt.cudaEventCreate())

    def flush_l2(i):
        ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))

    def device_step():
        _abi.check(lib.sb_refit_blas(ctx, root, end), ctx)
        _abi.check(lib.sb_update_transforms(ctx, None, None, 0), ctx)
        f.tick()

    # ---- counted run (untimed): traversal work of one step for the roofline
    _abi.check(lib.sb_enable_counters(ctx, 1), ctx)
    device_step()
    f.synchronize()
    st = _abi.sb_stats()
    _abi.check(lib.sb_get_stats(ctx, C.byref(st)), ctx)
    ray_data = np.zeros(rays * 4, np.float32)
    _abi.check(lib.sb_read_buffer(ctx, _abi.BUF["RAY_DATA"], 0, rays * 4, _abi.ptr(ray_data)), ctx)
    hits = int((ray_data[3::4] >= 0).sum())
    _abi.check(lib.sb_enable_counters(ctx, 0), ctx)
    counted = dict(primary=st.primaryRays, shadow=st.shadowRays, tlas=st.tlasNodeVisits, inst=st.instanceVisits,
                   blas=st.blasNodeVisits, tri=st.triangleTests, hits=hits,
                   shadow_tlas=st.shadowTlasNodeVisits, shadow_inst=st.shadowInstanceVisits,
                   shadow_blas=st.shadowBlasNodeVisits, shadow_tri=st.shadowTriangleTests)
    # algorithmic bytes per launch of each stage. Per-unit figures: 32 B TLAS node, 64 B instance
    # record, 48 B pre-gathered triangle; per box test 32 B (a BLAS node, or half a 64 B child-pair
    # node) or 10 B on the 8-wide closest-hit tree (80 B node / 8 boxes); 16 B raw hit record per ray
    # (written by the closest-hit stage, read by the emission stage); emission per ray 16 B visibility
    # mask, per hit 16 B final hit record + 48 B instance rows + 48 B pre-gathered triangle + 48 B
    # reference triangle (3 indices, 3 vertices) for the refined t, 32 B per shadow job (written by the
    # emission stage, read by the shadow stage); per hit 80 B of triangle/instance rows, 40 B material,
    # 256 B of bounce taps (8 taps x 4 texels x 8 B); 16 B ray record write; 3,776 B per probe for
    # blend + upload.
    tun = _abi.sb_tuning()
    _abi.check(lib.sb_get_tuning(ctx, C.byref(tun)), ctx)
    closest_box = 10 if tun.bvhKind == 1 else 32

    def trav(t, i, b, tr, box=32):
        return 32 * t + 64 * i + box * b + 48 * tr
    jobs = counted["shadow"]
    stage_bytes = {
        "k_trace_primary": trav(counted["tlas"] - counted["shadow_tlas"], counted["inst"] - counted["shadow_inst"],
                                counted["blas"] - counted["shadow_blas"], counted["tri"] - counted["shadow_tri"],
                                closest_box)
        + 16 * rays,
        "k_emit": 32 * rays + 160 * hits + 32 * jobs,
        "k_trace_shadow": trav(counted["shadow_tlas"], counted["shadow_inst"], counted["shadow_blas"],
                               counted["shadow_tri"]) + 32 * jobs,
        "k_shade": 48 * rays + 376 * hits,
        "k_blend_upload": 3776 * P,
    }
    trace_bytes = sum(stage_bytes.values())

    # ---- device-resident timed loop
    for i in range(W):
        device_step()
        flush_l2(i)
    f.synchronize()
    dist.barrier()
    clocks = Clocks(device)
    clocks.start()
    launches0 = _stats(lib, ctx).kernelLaunches
    total_ms = 0.0
    stage_ms = {k: [] for k in stage_bytes}
    for i in range(K):
        flush_l2(i)
        ck(rt.cudaEventRecord(e0, stream))
        device_step()
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        total_ms += ck(rt.cudaEventElapsedTime(e0, e1))
        s = _stats(lib, ctx)
        for k, v in (("k_trace_primary", s.lastPrimaryMs), ("k_emit", s.lastEmitMs),
                     ("k_trace_shadow", s.lastShadowMs), ("k_shade", s.lastShadeMs),
                     ("k_blend_upload", s.lastBlendMs)):
            stage_ms[k].append(v)
    launches = _stats(lib, ctx).kernelLaunches - launches0
    clk = clocks.stop()
    f.synchronize()
    ms_step = dist.max(total_ms / K)
    value = dist.world * rays / (ms_step * 1e-3) / 1e6

    # ---- e2e through the public facade (pinned host buffers)
    frames = [synth.atrium_motion(scene, fr) for fr in range(W + K)]
    r = f.getResolution()
    atl = _abi.PinnedArray((r[1] * r[2] * 8, r[0] * 8, 4), np.uint16)
    datl = _abi.PinnedArray((r[1] * r[2] * 8, r[0] * 8, 4), np.uint16)
    base_pos = scene.meshes[dm].positions

    def e2e_step(fr):
        mats, pos = frames[fr]
        scene.meshes[dm].positions = pos
        for i, m in mats.items():
            scene.instances[i].world = m
        f.markDeformsDirty()
        f.markTransformsDirty(list(mats))
        f.tick()
        f._debugReadMany([("atlas", atl.array), ("depthAtlas", datl.array)])

    for i in range(W):
        e2e_step(i)
        flush_l2(i)
    f.synchronize()
    dist.barrier()
    e2e_total = 0.0
    for i in range(K):
        flush_l2(i)
        ck(rt.cudaStreamSynchronize(stream))
        t0 = time.perf_counter()
        e2e_step(W + i)
        e2e_total += time.perf_counter() - t0
    e2e_ms = dist.max(e2e_total / K * 1e3)
    e2e_value = dist.world * rays / (e2e_ms * 1e-3) / 1e6
    # the deformer's positions (and normals, when the mesh has them) at 12 B per vertex each,
    # and per moved instance its FP64 4x4 matrix and source index
    h2d = base_pos.shape[0] * (12 if scene.meshes[dm].normals is None else 24) + len(movers) * (16 * 8 + 4)
    d2h = atl.array.nbytes + datl.array.nbytes
    scene.meshes[dm].positions = base_pos

    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    stage_avg = {k: sum(v) / len(v) for k, v in stage_ms.items()}
    dominant = max(stage_avg, key=stage_avg.get)
    achieved = stage_bytes[dominant] / (stage_avg[dominant] * 1e-3) / 1e9
    # DRAM bytes per launch from the committed ncu summary (lines "kernel bytes"); null when absent
    traffic = {}
    tf = ROOT / "profiles" / "dram_traffic.txt"
    if tf.exists():
        for ln in tf.read_text().splitlines():
            parts = ln.split()
            if len(parts) >= 2 and parts[0].startswith("k_") and parts[1].isdigit():
                traffic[parts[0]] = int(parts[1])
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist.world, "steps": K, "warmup": W,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded procedural atrium standing in for Sponza)",
        "config": atrium_config(P, f.getRays(), int(pool.triIndex.shape[0]), dist.world, args.reflection),
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "ms_per_step": round(e2e_ms, 4),
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic.get(dominant),
                     "algorithmic_bytes_per_launch": int(stage_bytes[dominant]),
                     "stage_ms": {k: round(v, 4) for k, v in stage_avg.items()},
                     "stage_gbs": {k: round(stage_bytes[k] / (stage_avg[k] * 1e-3) / 1e9, 1) for k in stage_avg
                                   if stage_avg[k] > 0},
                     "update_algorithmic_bytes": int(trace_bytes),
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback 6650 GB/s"},
        "work": {k: int(v) for k, v in counted.items()},
        "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(scene, target_s=12.0, reflection=args.reflection)
    f.dispose()
    ck(rt.cudaFree(flush))
    return line


def _stats(lib, ctx):
    from speedball_b200 import _abi
    st = _abi.sb_stats()
    _abi.check(lib.sb_get_stats(ctx, C.byref(st)), ctx)
    return st


# ----------------------------------------------------- CPU (reference arm)
class CpuAtrium:
    """The reference's own CPU path for one atrium update, built and run by the
    oracle alone (nothing here touches the CUDA library or its host code): the
    pool from the MeshBVH restatement, the TLAS and instance records from
    buildTlasRecords / computeDynamic, the uniforms at their defaults, the
    light selection of selectGiLightRecords. A step is the reference's per-frame
    work: updateDeforms (vertex gather + refitFlatBlasRange of the deforming
    mesh), updateTransforms (the 3 movers' instance rows + the TLAS refit of the
    frozen partition), then the FP32 solve of `probes` probes."""

    def __init__(self, scene, reflection: str = "off"):
        sys.path.insert(0, str(ROOT / "oracle"))
        import orc
        self.orc = orc
        self.lib = orc.load()
        self.scene = scene
        pool = self.pool = orc.OrcPool(scene)
        mats, order, live, aabb = orc.compute_tail(pool)
        self.mats, self.order = mats, order
        self.nodes = pool.bvhNodes
        self.vertex = pool.vertexData
        self.keep = [pool]
        self.S = orc.scene_struct(pool, mats, nodes=self.nodes, vertex=self.vertex, keep=self.keep)
        gm = scene.meta["grid"]
        self.g = orc.grid_dict(gm["gridMin"], gm["gridSize"], gm["res"], gm["rays"])
        gmax = [self.g["gridMin"][a] + self.g["gridSize"][a] for a in range(3)]
        recs, _, _ = orc.select_light_records(scene.lights, True, self.g["gridMin"], gmax)
        self.arena = orc.light_arena(recs, True, self.g)
        self.nl = recs.shape[0]
        self.prm = orc.default_params(scene.meta["hysteresis"])
        self.G = orc.grid_struct(self.g)
        self.irr, self.depth, self.atlas, self.datlas = orc.new_state(self.g, fp32=True)
        tier = orc.REFLECT_TIERS[reflection]
        self.rf = orc.ReflectState(self.g, tier, fp32=True) if tier else None
        self.probes = int(np.prod(self.g["res"]))
        self.dm = scene.meta["deformer"]
        self.movers = list(scene.meta["movers"])
        n = pool.instCount
        self.inv = np.zeros((n, 12), np.float32)
        self.det = np.zeros(n, np.float32)
        self.aabb = np.zeros((n, 9))
        self.world = pool.inst_world.copy()
        self.tl = np.ascontiguousarray(mats[pool.tlasBase:].copy())

    def lanes(self, frame_motion):
        """updateDeforms + updateTransforms of one frame on the host."""
        orc, lib, pool = self.orc, self.lib, self.pool
        mats_w, pos = frame_motion
        vb, vc = int(pool.vert_base[self.dm]), int(pool.vert_count[self.dm])
        self.vertex[vb:vb + vc, 0:3] = pos
        ok = lib.orc_refit_blas(orc._p(self.nodes), self.nodes.size, orc._p(pool.triIndex), pool.triIndex.size,
                                orc._p(self.vertex), self.vertex.size, int(pool.blas_root[self.dm]),
                                int(pool.blas_end[self.dm]))
        assert ok == 1
        for i, m in mats_w.items():
            self.world[i] = np.asarray(m, np.float64).T.reshape(16)
        lb = np.ascontiguousarray(orc.local_bounds(self.nodes, pool.inst_root))
        lib.orc_compute_instances(orc._p(self.world), orc._p(pool.inst_active), orc._p(lb), pool.instCount,
                                  orc._p(self.inv), orc._p(self.det), orc._p(self.aabb))
        ib = pool.instBase
        for slot, src in enumerate(self.order):
            self.mats[ib + slot * 28: ib + slot * 28 + 12] = self.inv[src]
            self.mats[ib + slot * 28 + 14] = self.det[src]
        live = np.ascontiguousarray(self.aabb[self.order, 0:6].astype(np.float32))
        assert lib.orc_refit_tlas_range(orc._p(self.tl), self.tl.size, orc._p(live), live.size, 0, pool.tlasNodeCount)
        self.mats[pool.tlasBase:] = self.tl

    def solve(self, probes: int, offset: int = 0):
        io = None
        if self.rf is not None:
            io = self.orc.OrcSolveIO()
            self.rf.attach(io)
        self.orc.solve(self.S, self.arena, self.nl, True, self.G, self.G, self.prm, offset, probes, self.irr,
                       self.depth, self.atlas, self.datlas, fp32=True, io=io)
        if self.rf is not None:
            self.rf.advance()

    def step(self, frame_motion, probes: int, offset: int = 0) -> float:
        t0 = time.perf_counter()
        self.lanes(frame_motion)
        self.solve(probes, offset)
        return time.perf_counter() - t0


def atrium_config(probes: int, rays: int, tris: int, world: int, reflection: str = "off") -> dict:
    """The workload description both arms print (the same keys and values)."""
    out = {"workload": "atrium 262,267 tris / 30 meshes, 16^3 probes x 64 rays, 32 clustered point + 1 "
                       "directional light, 1 deforming + 3 moving meshes per frame",
           "probes": probes, "rays_per_probe": rays, "primary_rays_per_step": probes * rays, "triangles": tris,
           "l2": "flushed (256 MiB write) before every timed step (GPU arm)",
           "parallelism": "replicas" if world > 1 else "single GPU"}
    if reflection != "off":
        out["reflection"] = reflection
    return out


def cpu_baseline(scene, target_s=12.0, reflection="off"):
    """The FP32 CPU restatement on every host thread: whole-atrium updates (the
    motion lanes + all 4,096 probes) repeated for about `target_s` seconds."""
    from speedball_b200 import synth
    threads = os.cpu_count() or 1
    cpu = CpuAtrium(scene, reflection)
    dt = cpu.step(synth.atrium_motion(scene, 0), cpu.probes)
    reps = max(1, int(round(target_s / max(dt, 1e-3))))
    frames = [synth.atrium_motion(scene, 1 + i) for i in range(reps)]
    total = sum(cpu.step(fr, cpu.probes) for fr in frames)
    rate = cpu.probes * cpu.g["rays"] * reps / total / 1e6
    return {"value": round(rate, 4), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{reps} full atrium updates (deformer refit + 3 movers + TLAS refit + 4,096 probes x 64 rays) "
                      f"on {threads} threads, FP32 CPU restatement built by the oracle alone, {total:.1f} s"}


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return None
    from speedball_b200 import synth
    scene = make_workload()
    threads = os.cpu_count() or 1
    cpu = CpuAtrium(scene, args.reflection)
    W, K = args.warmup, args.steps
    frames = [synth.atrium_motion(scene, fr) for fr in range(W + K + 1)]
    dt = cpu.step(frames[-1], cpu.probes)
    # each step a whole-atrium update, or a probe sample sized so the K + W steps fit about 2 minutes
    budget_s = 120.0
    per_step = budget_s / max(1, K + W)
    probes = int(min(cpu.probes, max(64, cpu.probes * per_step / max(dt, 1e-3))))
    for i in range(W):
        cpu.step(frames[i], probes)
    total = 0.0
    offset = 0
    for i in range(K):
        total += cpu.step(frames[W + i], probes, offset)
        offset = (offset + probes) % cpu.probes
    value = K * probes * cpu.g["rays"] / total / 1e6
    rays = cpu.probes * cpu.g["rays"]
    sample = (f"{probes} of {cpu.probes} probes x 64 rays per step, with the step's deformer refit, 3 movers and "
              f"TLAS refit; FP32 CPU restatement of the reference path built by the oracle alone, {threads} threads "
              "(the reference itself is WebGPU/JS: no runtime here)")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": dist.world,
            "steps": K, "warmup": W, "ms_per_step": round(rays / (value * 1e6) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural atrium standing in for Sponza)",
            "config": atrium_config(cpu.probes, cpu.g["rays"], int(cpu.pool.triIndex.shape[0]), dist.world,
                                    args.reflection),
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


ADJ_METRIC = "adjoint / forward device time"


def adjoint_field(device):
    from speedball_b200 import synth
    from speedball_b200.field import ProbeField
    scene = synth.room_spheres(0, n_materials=64, n_point=32, n_dir=0)
    g = scene.meta["grid"]
    f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1, rays=g["rays"],
                   hysteresis=scene.meta["hysteresis"], jitterMode="gated", device=device)
    f.setHysteresisNormalization(False)
    f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
    return scene, f


def run_adjoint(args, dist: Dist):
    """One step = one gradient evaluation: sb_forward_record (2 feedback solves
    from a cleared history, tape, loss) + sb_backward (re-shade + reverse
    kernels), 416 parameters. value = backward device time / forward-record
    device time; the plain forward (the same 2 solves, nothing recorded) is
    timed beside it."""
    from speedball_b200 import _abi
    from speedball_b200.adjoint import GIAdjoint
    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    scene, f = adjoint_field(device)
    lib, ctx = f._lib, f.ctx
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    _abi.check(lib.sb_set_stream(ctx, C.c_void_p(int(stream))), ctx)
    flush = ck(rt.cudaMalloc(L2_FLUSH_BYTES))
    adj = GIAdjoint(f, solves=2)
    rng = np.random.default_rng(7)
    base = adj.parameters()
    adj.setParameters(albedo=base["albedo"] * rng.uniform(0.8, 1.2, (64, 3)), lightScale=rng.uniform(0.5, 2.0, 32))
    target = _abi.PinnedArray((adj.probes, 36, 3), np.float32)
    target.array[...] = adj.forward()
    adj.setParameters(albedo=base["albedo"], lightScale=np.ones(32))
    W, K = args.warmup, args.steps
    e0, e1 = ck(rt.cudaEventCreate()), ck(rt.cudaEventCreate())

    def flush_l2(i):
        ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
        ck(rt.cudaStreamSynchronize(stream))

    def plain_forward():
        # the same two solves without the tape (their work does not depend on
        # the history they start from)
        for _ in range(2):
            _abi.check(lib.sb_solve(ctx, 0, 0, adj.probes), ctx)

    for i in range(W):
        adj.forward(target.array)
        adj.backward()
        flush_l2(i)
    dist.barrier()
    clocks = Clocks(device)
    clocks.start()
    launches0 = _stats(lib, ctx).kernelLaunches
    fwd, bwd, wall = [], [], []
    for i in range(K):
        flush_l2(i)
        t0 = time.perf_counter()
        adj.forward(target.array)
        adj.backward()
        wall.append(time.perf_counter() - t0)
        tm = adj.timings()
        fwd.append(tm["forwardMs"])
        bwd.append(tm["backwardMs"])
    launches = _stats(lib, ctx).kernelLaunches - launches0
    plain = []
    for i in range(K):
        flush_l2(i)
        ck(rt.cudaEventRecord(e0, stream))
        plain_forward()
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        plain.append(ck(rt.cudaEventElapsedTime(e0, e1)))
    clk = clocks.stop()
    fwd_ms, bwd_ms = dist.max(statistics.mean(fwd)), dist.max(statistics.mean(bwd))
    plain_ms = dist.max(statistics.mean(plain))
    wall_ms = dist.max(statistics.mean(wall) * 1e3)
    nparam = 6 * adj.materialCount + adj.lightCount
    line = {
        "metric": ADJ_METRIC, "value": round(bwd_ms / fwd_ms, 4), "unit": "x", "n_gpus": dist.world, "steps": K,
        "warmup": W, "ms_per_step": round(fwd_ms + bwd_ms, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded room + 64 icospheres)",
        "config": {"workload": "differentiated update: room + 64 icospheres (81,932 tris), 64 materials, 32 point "
                               "lights, 8^3 probes x 64 rays, 2 feedback solves, 416 parameters",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "forward_record_ms": round(fwd_ms, 4), "backward_ms": round(bwd_ms, 4),
        "plain_forward_ms": round(plain_ms, 4), "backward_over_plain_forward": round(bwd_ms / plain_ms, 4),
        "e2e": {"value": round(wall_ms / plain_ms, 4), "unit": "x (gradient wall time / plain forward device time)",
                "ms_per_step": round(wall_ms, 4), "h2d_bytes_per_step": int(target.array.nbytes),
                "d2h_bytes_per_step": int(8 + nparam * 8)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_adjoint_baseline(f, adj, target.array)
    f.dispose()
    ck(rt.cudaFree(flush))
    return line


def cpu_adjoint_baseline(f, adj, target):
    """The oracle's FP64 adjoint (forward + reverse pass) of the same gradient
    on every host thread, replaying the GPU's hit records."""
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    from gpu_util import OracleMirror, gpu_records
    import orc
    mirror = OracleMirror(f)
    rec = gpu_records(f, adj.probes * f.getRays())
    base = adj.parameters()
    t0 = time.perf_counter()
    orc.adjoint(mirror.scene, mirror.arena, mirror.light_count, mirror.clustered, mirror.grid, mirror.params(),
                rec["tri"], rec["inst_word"], rec["blocked"], 2, base["albedo"].reshape(-1),
                base["emissive"].reshape(-1), np.ones(adj.lightCount), target=target.astype(np.float64).reshape(-1))
    dt = time.perf_counter() - t0
    return {"value": round(dt * 1e3, 2), "unit": "ms per gradient", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": "one FP64 oracle gradient (2 solves forward + reverse, 416 parameters) on all host threads"}


BATCH_METRIC = "batched probe Mrays/s (11 solves per frame)"


def batch_fields(device):
    """The atrium with 3 nested cascades (16^3, 12^3, 8^3; each twice the
    previous extent) and 8 independent atria of 20k-500k triangles with their
    own grids and ray counts, montecarlo jitter, full updates every frame."""
    from speedball_b200 import synth
    from speedball_b200.field import ProbeField

    def make(scene, jitter):
        g = scene.meta["grid"]
        f = ProbeField(scene, volumes=dict(gridMin=g["gridMin"], gridSize=g["gridSize"], res=g["res"]), cascades=1,
                       rays=g["rays"], clusteredLighting=True, hysteresis=scene.meta["hysteresis"],
                       jitterMode=jitter, device=device)
        f.setHysteresisNormalization(False)
        f.setRayBudget(1 << 24, maxProbesPerTick=1 << 20)
        return f

    main_scene = make_workload()
    fields = [make(main_scene, "montecarlo")]
    for ci, c in enumerate(synth.nested_cascades(main_scene.meta["grid"])[1:], start=1):
        fields[0].configureCascade(ci, c["gridMin"], c["gridSize"], c["res"])
    scenes = [main_scene] + synth.batch_scenes()
    fields += [make(s, "montecarlo") for s in scenes[1:]]
    return scenes, fields


def run_batch(args, dist: Dist):
    """One step = one frame: every scene's motion lanes on the device (deformer
    refit, instance bounds + TLAS refit) and 11 solves (the atrium's 3
    cascades, the 8 atria's C0), after sb_autotune on every context. value =
    primary rays / device time of the frame as one CUDA graph (lanes as
    parallel branches, one batched solve); beside it the same frames as
    ordinary batched launches and as per-solve launches (the plain form)."""
    from speedball_b200 import _abi
    from speedball_b200.batch import BatchedFrame
    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    scenes, fields = batch_fields(device)
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    frame = BatchedFrame(fields, extra=[(fields[0], 1), (fields[0], 2)])
    frame.setStream(int(stream))
    flush = ck(rt.cudaMalloc(L2_FLUSH_BYTES))
    lanes = []
    for s, f in zip(scenes, fields):
        dm = s.meta["deformer"]
        lanes.append((f, int(f.pool.blas_root[dm]), int(f.pool.blas_end[dm])))
    rays = sum(f._probeTotal * f.getRays() for f in fields)
    rays += sum(fields[0].cascadeProbes(ci) * fields[0].getRays() for ci in (1, 2))
    tris = sum(int(f.pool.triIndex.shape[0]) for f in fields)
    W, K = args.warmup, args.steps
    e0, e1 = ck(rt.cudaEventCreate()), ck(rt.cudaEventCreate())

    def motion():
        for f, root, end in lanes:
            _abi.check(f._lib.sb_refit_blas(f.ctx, root, end), f.ctx)
            _abi.check(f._lib.sb_update_transforms(f.ctx, None, None, 0), f.ctx)

    def timed(step):
        for i in range(W):
            step()
            ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
        ck(rt.cudaStreamSynchronize(stream))
        dist.barrier()
        l0 = _stats(fields[0]._lib, fields[0].ctx).kernelLaunches
        total = 0.0
        for i in range(K):
            ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
            ck(rt.cudaEventRecord(e0, stream))
            step()
            ck(rt.cudaEventRecord(e1, stream))
            ck(rt.cudaEventSynchronize(e1))
            total += ck(rt.cudaEventElapsedTime(e0, e1))
        launches = _stats(fields[0]._lib, fields[0].ctx).kernelLaunches - l0
        return dist.max(total / K), launches

    def batched():
        motion()
        frame.tick()

    def plain():
        motion()
        frame.tickPlain()

    from speedball_b200.batch import GraphFrame, Lane, autotune
    # every context gets its autotuned traversal parameters (plain and batched
    # frames alike; the batch runs with the lead context's block size and ray
    # order, and each scene's own BVH kind)
    t0 = time.perf_counter()
    tunings = [autotune(f) for f in fields]
    tune_s = time.perf_counter() - t0
    graph = GraphFrame(frame, [Lane(f, [(root, end)]) for f, root, end in lanes])

    clocks = Clocks(device)
    clocks.start()
    ms_plain, _ = timed(plain)
    from speedball_b200.batch import autotuneBatch
    full = [dict(cascade=0, probeOffset=0, updatedCount=f._probeTotal) for f in fields]
    t0 = time.perf_counter()
    batch_tuning = autotuneBatch(frame.items(full))
    tune_s += time.perf_counter() - t0
    ms_nograph, _ = timed(batched)
    ms_batch, launches = timed(graph.tick)
    clk = clocks.stop()
    graph.dispose()
    value = dist.world * rays / (ms_batch * 1e-3) / 1e6
    plain_value = dist.world * rays / (ms_plain * 1e-3) / 1e6
    line = {
        "metric": BATCH_METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": dist.world, "steps": K,
        "warmup": W, "ms_per_step": round(ms_batch, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural atria)",
        "config": {"workload": "atrium 262,267 tris with 3 nested cascades (16^3, 12^3, 8^3 probes x 64 rays; "
                               "extents x1, x2, x4) + 8 atria of 20k-500k tris with 8^3-16^3 probes at 32-128 "
                               "rays; montecarlo jitter; per frame every scene's deformer refit + TLAS refit",
                   "solves_per_frame": 11, "primary_rays_per_step": int(rays), "triangles": tris,
                   "grids": [list(f.getResolution()) + [f.getRays()] for f in fields],
                   "l2": "flushed (256 MiB write) before every timed step"},
        "plain_value": round(plain_value, 3), "plain_ms_per_step": round(ms_plain, 4),
        "batched_no_graph_ms_per_step": round(ms_nograph, 4),
        "autotuned": tunings, "autotuned_batch": batch_tuning, "autotune_s": round(tune_s, 2),
        "batched_over_plain": round(ms_plain / ms_batch, 4),
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    for f in fields:
        f.dispose()
    ck(rt.cudaFree(flush))
    return line


GATHER_METRIC = "receiver gather Msamples/s (1920x1080 G-buffer)"


def camera_gbuffer(f, scene, width=1920, height=1080):
    """A deferred G-buffer of the atrium from a pinhole camera at the probe
    grid's centre looking along +x (90 degree horizontal field of view): per
    covered pixel the hit position and the geometric world normal facing the
    camera (sky pixels dropped, as a deferred pass skips them). float4 rows."""
    from speedball_b200 import _abi
    g = scene.meta["grid"]
    c = np.asarray(g["gridMin"], np.float64) + 0.5 * np.asarray(g["gridSize"], np.float64)
    xs = (np.arange(width) + 0.5) / width * 2 - 1
    ys = ((np.arange(height) + 0.5) / height * 2 - 1) * height / width
    X, Y = np.meshgrid(xs, ys)
    d = np.stack([np.ones_like(X), -Y, X], -1).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    n = d.shape[0]
    ro = np.ascontiguousarray(np.broadcast_to(c, (n, 3)), np.float32)
    rd = np.ascontiguousarray(d, np.float32)
    t = np.zeros(n, np.float32)
    tri = np.zeros(n, np.int32)
    slot = np.zeros(n, np.int32)
    _abi.check(f._lib.sb_raycast(f.ctx, _abi.ptr(ro), _abi.ptr(rd), n, _abi.ptr(t), _abi.ptr(tri), _abi.ptr(slot)),
               f.ctx)
    hit = tri >= 0
    pool = f.pool
    order = np.zeros(pool.instCount, np.uint32)
    _abi.check(f._lib.sb_read_buffer(f.ctx, _abi.BUF["TLAS_ORDER"], 0, pool.instCount, _abi.ptr(order)), f.ctx)
    src = order[slot[hit]]
    idx = pool.triIndex[tri[hit]]
    v = pool.vertexData[:, 0:3].astype(np.float64)
    p0, p1, p2 = v[idx[:, 0]], v[idx[:, 1]], v[idx[:, 2]]
    nl = np.cross(p1 - p0, p2 - p0)
    W = np.stack([scene.instances[i].world for i in range(pool.instCount)])[src]
    Minv = np.linalg.inv(W[:, :3, :3])
    nw = np.einsum("nji,nj->ni", Minv, nl)  # (M^-1)^T n
    nw /= np.linalg.norm(nw, axis=1, keepdims=True)
    dh = d[hit]
    nw *= np.where(np.einsum("ni,ni->n", nw, dh) > 0, -1.0, 1.0)[:, None]
    m = int(hit.sum())
    pos = np.zeros((m, 4), np.float32)
    pos[:, :3] = ro[hit] + rd[hit] * t[hit, None]
    nrm = np.zeros((m, 4), np.float32)
    nrm[:, :3] = nw
    return pos, nrm


def run_gather(args, dist: Dist):
    """One step = one receiver gather of a 1920x1080 deferred G-buffer of the
    atrium (covered pixels) from the atlases of 4 updates: position, stable
    normal and detail normal in (48 B per sample), irradiance out (16 B).
    With --reflection rough / high / ultra the step is the combined receiver
    (sb_gather_reflections) on that tier's atlases: the mirror reflection of
    the camera ray about the normal and a seeded roughness in [0, 1) also in
    (16 B), the reflection layer also out (16 B).
    value = samples / device time; e2e = the same through host buffers
    (G-buffer up, outputs down, page-locked)."""
    from speedball_b200 import _abi
    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    scene = make_workload()
    combined = args.reflection != "off"
    f = field_for(scene, device, args.reflection)
    for _ in range(4):
        f.tick()
    f.synchronize()
    pos, nrm = camera_gbuffer(f, scene)
    n = pos.shape[0]
    inputs = [pos, nrm, nrm]
    if combined:
        g = scene.meta["grid"]
        cam = np.asarray(g["gridMin"], np.float64) + 0.5 * np.asarray(g["gridSize"], np.float64)
        v = pos[:, :3].astype(np.float64) - cam
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        nn = nrm[:, :3].astype(np.float64)
        refl = np.zeros((n, 4), np.float32)
        refl[:, :3] = v - 2.0 * np.einsum("ni,ni->n", v, nn)[:, None] * nn
        refl[:, 3] = np.random.default_rng(31).uniform(0.0, 1.0, n)
        inputs.append(refl)
    n_out = 2 if combined else 1
    lib, ctx = f._lib, f.ctx
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    _abi.check(lib.sb_set_stream(ctx, C.c_void_p(int(stream))), ctx)
    flush = ck(rt.cudaMalloc(L2_FLUSH_BYTES))
    bufs = [ck(rt.cudaMalloc(n * 16)) for _ in range(len(inputs) + n_out)]
    for b, a in zip(bufs, inputs):
        ck(rt.cudaMemcpy(b, a.ctypes.data, n * 16, rt.cudaMemcpyKind.cudaMemcpyHostToDevice))
    prm = _abi.sb_gather_params()
    lib.sb_gather_params_defaults(C.byref(prm))
    prm.normalBias[0] = max(1e-4, f.grid.cellMin * 0.04)
    ptr = [C.c_void_p(int(b)) for b in bufs]

    def gather():
        if combined:
            _abi.check(lib.sb_gather_reflections(ctx, C.byref(prm), ptr[0], ptr[1], ptr[2], ptr[3], n, ptr[4],
                                                 ptr[5]), ctx)
        else:
            _abi.check(lib.sb_gather_irradiance(ctx, C.byref(prm), ptr[0], ptr[1], ptr[2], n, ptr[3]), ctx)

    e0, e1 = ck(rt.cudaEventCreate()), ck(rt.cudaEventCreate())
    W, K = args.warmup, args.steps
    for i in range(W):
        ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
        gather()
    ck(rt.cudaStreamSynchronize(stream))
    dist.barrier()
    clocks = Clocks(device)
    clocks.start()
    total = 0.0
    for i in range(K):
        ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
        ck(rt.cudaEventRecord(e0, stream))
        gather()
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        total += ck(rt.cudaEventElapsedTime(e0, e1))
    ms = dist.max(total / K)
    # end to end: page-locked G-buffer up, gather, outputs down
    hp = [_abi.PinnedArray((n, 4), np.float32) for _ in range(len(bufs))]
    for h, a in zip(hp, inputs):
        h.array[...] = a
    H2D, D2H = rt.cudaMemcpyKind.cudaMemcpyHostToDevice, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost
    e2e = 0.0
    for i in range(W + K):
        ck(rt.cudaStreamSynchronize(stream))
        t0 = time.perf_counter()
        for b, h in zip(bufs[:len(inputs)], hp[:len(inputs)]):
            ck(rt.cudaMemcpyAsync(b, h.array.ctypes.data, n * 16, H2D, stream))
        gather()
        for b, h in zip(bufs[len(inputs):], hp[len(inputs):]):
            ck(rt.cudaMemcpyAsync(h.array.ctypes.data, b, n * 16, D2H, stream))
        ck(rt.cudaStreamSynchronize(stream))
        if i >= W:
            e2e += time.perf_counter() - t0
    e2e_ms = dist.max(e2e / K * 1e3)
    clk = clocks.stop()
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    bytes_per = 16.0 * len(bufs)
    achieved = bytes_per * n / (ms * 1e-3) / 1e9
    out = hp[len(inputs)].array
    line = {
        "metric": GATHER_METRIC, "value": round(dist.world * n / (ms * 1e-3) / 1e6, 2), "unit": "Msamples/s",
        "n_gpus": dist.world, "steps": K, "warmup": W, "ms_per_step": round(ms, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (RGBA16F atlases)",
        "data": "synthetic (seeded procedural atrium, atlases of 4 updates)",
        "config": {"workload": ("combined receiver (irradiance + reflection layer, reflection tier "
                                f"{args.reflection})" if combined else "receiver gather") +
                               " of a 1920x1080 deferred G-buffer of the atrium (covered pixels), 16^3 probes, "
                               "default receiver uniforms (8-tap trilinear)", "samples": n,
                   "l2": "flushed (256 MiB write) before every timed step"},
        "e2e": {"value": round(dist.world * n / (e2e_ms * 1e-3) / 1e6, 2), "unit": "Msamples/s",
                "ms_per_step": round(e2e_ms, 4), "h2d_bytes_per_step": 16 * len(inputs) * n,
                "d2h_bytes_per_step": 16 * n_out * n},
        "gpu_launches": K,
        "roofline": {"bound": "hbm", "kernel": "k_gather_combined" if combined else "k_gather",
                     "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": int(bytes_per * n),
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback 6650 GB/s"},
        "irradiance_mean": [round(float(x), 5) for x in out[:, :3].mean(0)],
        "clocks": clk,
    }
    if combined:
        r = hp[len(inputs) + 1].array
        line["reflection_mean"] = [round(float(x), 5) for x in r.mean(0)]
    for b in bufs:
        ck(rt.cudaFree(b))
    ck(rt.cudaFree(flush))
    f.dispose()
    return line


BUILD_METRIC = "BLAS build Mtris/s (GPU linear BVH, threaded layout)"


def run_build(args, dist: Dist):
    """One step = the BLAS builds of every mesh of the atrium (30 meshes,
    262,267 triangles) and of the large scene's 8 archetypes (2.1M triangles)
    on the GPU (sb_build_blas_device: device arrays in, threaded nodes out),
    the meshes resident in HBM. Beside it, once per mesh on the host: the
    library's host builder and the oracle's MeshBVH restatement (the
    reference's CPU build)."""
    from speedball_b200 import _abi, synth
    from speedball_b200 import scene as sc
    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    lib = _abi.load()
    h = C.c_void_p()
    _abi.check(lib.sb_create(C.byref(_abi.sb_device_opts(device, 0)), C.byref(h)))
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    _abi.check(lib.sb_set_stream(h, C.c_void_p(int(stream))), h)
    meshes = synth.atrium(1).meshes + synth.large_scene().meshes
    H2D = rt.cudaMemcpyKind.cudaMemcpyHostToDevice
    dev = []
    for m in meshes:
        pos = np.ascontiguousarray(m.positions, np.float32)
        idx = np.ascontiguousarray(m.indices, np.uint32)
        T = idx.shape[0]
        bufs = [ck(rt.cudaMalloc(pos.nbytes)), ck(rt.cudaMalloc(idx.nbytes)), ck(rt.cudaMalloc(T * 64)),
                ck(rt.cudaMalloc(T * 4)), ck(rt.cudaMalloc(4))]
        ck(rt.cudaMemcpy(bufs[0], pos.ctypes.data, pos.nbytes, H2D))
        ck(rt.cudaMemcpy(bufs[1], idx.ctypes.data, idx.nbytes, H2D))
        dev.append((pos.shape[0], T, bufs))
    tris = sum(T for _, T, _ in dev)

    def step():
        for V, T, b in dev:
            _abi.check(lib.sb_build_blas_device(h, C.c_void_p(int(b[0])), V, C.c_void_p(int(b[1])), T, 8,
                                                C.c_void_p(int(b[2])), C.c_void_p(int(b[3])), C.c_void_p(int(b[4]))),
                       h)

    e0, e1 = ck(rt.cudaEventCreate()), ck(rt.cudaEventCreate())
    W, K = args.warmup, args.steps
    for _ in range(W):
        step()
    ck(rt.cudaStreamSynchronize(stream))
    clocks = Clocks(device)
    clocks.start()
    total = 0.0
    l0 = _stats(lib, h).kernelLaunches
    for _ in range(K):
        ck(rt.cudaEventRecord(e0, stream))
        step()
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        total += ck(rt.cudaEventElapsedTime(e0, e1))
    clk = clocks.stop()
    launches = _stats(lib, h).kernelLaunches - l0
    _abi.check(lib.sb_synchronize(h), h)
    ms = dist.max(total / K)
    # the largest mesh alone
    big = max(range(len(dev)), key=lambda i: dev[i][1])
    V, T, b = dev[big]
    tb = 0.0
    for _ in range(K):
        ck(rt.cudaEventRecord(e0, stream))
        _abi.check(lib.sb_build_blas_device(h, C.c_void_p(int(b[0])), V, C.c_void_p(int(b[1])), T, 8,
                                            C.c_void_p(int(b[2])), C.c_void_p(int(b[3])), C.c_void_p(int(b[4]))), h)
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        tb += ck(rt.cudaEventElapsedTime(e0, e1))
    big_ms = tb / K
    # host builders on the same meshes, once
    t0 = time.perf_counter()
    for m in meshes:
        sc.build_blas(m)
    host_ms = (time.perf_counter() - t0) * 1e3
    sys.path.insert(0, str(ROOT / "oracle"))
    import orc
    t0 = time.perf_counter()
    for m in meshes:
        orc.build_blas(m.positions, m.indices)
    orc_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    orc.build_blas(meshes[big].positions, meshes[big].indices)
    orc_big_ms = (time.perf_counter() - t0) * 1e3
    for _, _, bufs in dev:
        for p in bufs:
            ck(rt.cudaFree(p))
    lib.sb_destroy(h)
    line = {
        "metric": BUILD_METRIC, "value": round(dist.world * tris / (ms * 1e-3) / 1e6, 2), "unit": "Mtris/s",
        "n_gpus": dist.world, "steps": K, "warmup": W, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 bounds, u32 keys",
        "data": "synthetic (the atrium's 30 meshes + the large scene's 8 archetypes)",
        "config": {"workload": f"BLAS builds of {len(dev)} meshes, {tris} triangles, leaves of <= 8", "meshes": len(dev),
                   "triangles": int(tris)},
        "largest_mesh": {"triangles": int(T), "gpu_ms": round(big_ms, 4), "oracle_meshbvh_ms": round(orc_big_ms, 1)},
        "host_builder_ms_all": round(host_ms, 1), "oracle_meshbvh_ms_all": round(orc_ms, 1),
        "cpu_baseline": {"value": round(tris / (orc_ms * 1e-3) / 1e6, 3), "unit": "Mtris/s", "cores": 1,
                         "kind": "port", "sample": "the oracle's MeshBVH restatement (one thread) on every mesh once"},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    return line


LARGE_METRIC = "probe Mrays/s (large scene, 2 cascades)"


def large_field(device):
    """The large scene's field: 32^3 probes x 256 rays over the world box, and
    the fine cascade C1 that fitFineBox places inside it (the reference's
    two-cascade install, divisions 32 so that C1 may reach the 32-per-axis
    cap); clustered lights, gated jitter, full updates."""
    from speedball_b200 import synth
    scene = synth.large_scene()
    return scene, synth.large_field(scene, device=device)


def run_large(args, dist: Dist):
    """One step = one frame: the skinned mesh posed (bone rotations <= 15 deg),
    its vertices uploaded from page-locked memory, its BLAS refit, instance
    bounds + TLAS refit, then full solves of both cascades (16.8M primary
    rays). Timed once per scene-BVH layout: bvhKind 2 (binary, FP32 boxes),
    1 (8-wide, 8-bit boxes for closest hits) and 0 (the reference's TLAS +
    BLAS walk); hit records of the layouts are compared on a fixed pose."""
    from speedball_b200 import _abi, synth
    device = dist.local
    rt = cudart()
    ck(rt.cudaSetDevice(device))
    t0 = time.perf_counter()
    scene, f = large_field(device)
    setup_s = time.perf_counter() - t0
    lib, ctx = f._lib, f.ctx
    stream = ck(rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking))
    _abi.check(lib.sb_set_stream(ctx, C.c_void_p(int(stream))), ctx)
    flush = ck(rt.cudaMalloc(L2_FLUSH_BYTES))
    sk = scene.meta["skinned"]
    W, K = args.warmup, args.steps
    poses = [synth.large_pose(scene, fr) for fr in range(W + K + 1)]
    rays = (f._probeTotal + f.cascadeProbes(1)) * f.getRays()
    e0, e1 = ck(rt.cudaEventCreate()), ck(rt.cudaEventCreate())

    def frame(i):
        scene.meshes[sk].positions = poses[i]
        f.refreshDeforms([sk])           # pinned upload + BLAS refit + TLAS refit
        fr = f.beginTick()
        _abi.check(lib.sb_solve(ctx, 0, fr["probeOffset"], fr["updatedCount"]), ctx)
        _abi.check(lib.sb_solve(ctx, 1, 0, f.cascadeProbes(1)), ctx)
        f.endTick(fr)

    def hits(ci):
        n = f.cascadeProbes(ci) * f.getRays()
        h = np.zeros(n * 4, np.uint32)
        _abi.check(lib.sb_read_buffer(ctx, _abi.BUF["HIT_RECORDS"] | (ci << 8), 0, n * 4, _abi.ptr(h)), ctx)
        return h.reshape(n, 4)

    results, records = {}, {}
    clocks = Clocks(device)
    clocks.start()
    launches = 0
    for kind in (2, 1, 0):
        t = _abi.sb_tuning()
        _abi.check(lib.sb_get_tuning(ctx, C.byref(t)), ctx)
        t.bvhKind = kind
        _abi.check(lib.sb_set_tuning(ctx, C.byref(t)), ctx)
        tb = time.perf_counter()
        for i in range(W):
            frame(i)
            ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
        f.synchronize()
        warm_s = time.perf_counter() - tb
        dist.barrier()
        l0 = _stats(lib, ctx).kernelLaunches
        total = 0.0
        for i in range(K):
            ck(rt.cudaMemsetAsync(flush, i & 0xFF, L2_FLUSH_BYTES, stream))
            ck(rt.cudaEventRecord(e0, stream))
            frame(W + i)
            ck(rt.cudaEventRecord(e1, stream))
            ck(rt.cudaEventSynchronize(e1))
            total += ck(rt.cudaEventElapsedTime(e0, e1))
        launches += _stats(lib, ctx).kernelLaunches - l0
        ms = dist.max(total / K)
        frame(W + K)                      # the same pose for every layout: compare hit records
        f.synchronize()
        records[kind] = (hits(0), hits(1))
        results[kind] = {"ms_per_step": round(ms, 3), "mrays_s": round(dist.world * rays / (ms * 1e-3) / 1e6, 2),
                         "warmup_s": round(warm_s, 2)}
    # a structural rebuild of the bvhKind 1 trees: blocking (inside the next frame), then in
    # background mode, where frames go on with the two-level walk until the tree is installed
    t = _abi.sb_tuning()
    _abi.check(lib.sb_get_tuning(ctx, C.byref(t)), ctx)
    t.bvhKind = 1
    _abi.check(lib.sb_set_tuning(ctx, C.byref(t)), ctx)  # a layout change: the trees are rebuilt
    tb = time.perf_counter()
    frame(0)
    f.synchronize()
    blocking_frame_s = time.perf_counter() - tb
    blocking_build_ms = _stats(lib, ctx).lastSceneBvhBuildMs
    _abi.check(lib.sb_set_scene_bvh_build_mode(ctx, 1), ctx)
    _abi.check(lib.sb_rebuild_scene_bvh(ctx), ctx)
    during, n, tb = [], 0, time.perf_counter()
    while True:
        ck(rt.cudaEventRecord(e0, stream))
        frame(n % (W + K))
        ck(rt.cudaEventRecord(e1, stream))
        ck(rt.cudaEventSynchronize(e1))
        n += 1
        s = _stats(lib, ctx)
        if s.sceneBvhActive or time.perf_counter() - tb > 300.0:
            break
        during.append(ck(rt.cudaEventElapsedTime(e0, e1)))
    background = {"frames_before_install": len(during), "installed": bool(s.sceneBvhActive),
                  "ms_per_frame_while_building": round(float(np.mean(during)), 3) if during else None,
                  "max_frame_ms_while_building": round(float(np.max(during)), 3) if during else None,
                  "build_s": round(s.lastSceneBvhBuildMs / 1e3, 2), "wall_s": round(time.perf_counter() - tb, 2)}
    _abi.check(lib.sb_set_scene_bvh_build_mode(ctx, 0), ctx)
    clk = clocks.stop()

    def agree(a, b):
        same = (a[:, 0] == b[:, 0]) & ((a[:, 1] & 0x7FFFFFFF) == (b[:, 1] & 0x7FFFFFFF))
        t_a, t_b = a[:, 2].view(np.float32), b[:, 2].view(np.float32)
        hit = a[:, 0] != 0xFFFFFFFF
        rel = np.abs(t_a - t_b) / np.maximum(np.abs(t_a), 1e-30)
        return {"hit_id_agreement": round(float(same.mean()), 7),
                "t_rel_max_where_ids_agree": float(rel[same & hit].max()) if (same & hit).any() else 0.0,
                "differing_rays": int((~same).sum())}
    cmp = {f"kind{k}_vs_kind2": {f"c{ci}": agree(records[k][ci], records[2][ci]) for ci in (0, 1)} for k in (1, 0)}
    best = min(results, key=lambda k: results[k]["ms_per_step"])
    line = {
        "metric": LARGE_METRIC, "value": results[1]["mrays_s"], "unit": "Mrays/s", "n_gpus": dist.world, "steps": K,
        "warmup": W, "ms_per_step": results[1]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded large instanced scene)",
        "config": {"workload": "8 archetypes of 2k-600k tris (2,101,000 unique), 400 instances (12,810,000 "
                               "instanced), a 120k-tri skinned tube refit every frame (8 bones, <=15 deg), 64 "
                               "clustered point lights, C0 32^3 probes + the fitted fine cascade C1 (fitFineBox), 256 rays",
                   "c1": {"res": [int(f._c1Grid.res[a]) for a in range(3)] if f.hasFineCascade() else None,
                          "gridMin": [round(v, 4) for v in f._c1Box[0]] if f.hasFineCascade() else None,
                          "gridSize": [round(v, 4) for v in f._c1Box[1]] if f.hasFineCascade() else None},
                   "primary_rays_per_step": int(rays), "layout_of_value": "bvhKind 1 (8-wide, 8-bit boxes)",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "layouts": {f"bvhKind{k}": v for k, v in results.items()}, "fastest_layout": f"bvhKind{best}",
        "hit_agreement": cmp, "setup_s": round(setup_s, 2),
        "scene_bvh_rebuild": {"blocking_frame_s": round(blocking_frame_s, 2),
                              "blocking_build_s": round(blocking_build_ms / 1e3, 2), "background": background},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    f.dispose()
    ck(rt.cudaFree(flush))
    return line


def aux_measurements(args, dist: Dist) -> dict:
    """The batched form's and the adjoint's ratios, measured in the same run
    as the headline (each its own workload, set-up outside its timed region):
    `batch` = the 9-scene batched frame against the same frame as per-solve
    launches (target >= 3x), `adjoint` = backward / forward-record device time
    (target <= 3x)."""
    import types
    sub = types.SimpleNamespace(**vars(args))
    sub.steps = min(args.steps, 50)
    sub.warmup = max(3, min(args.warmup, 5))
    sub.no_cpu_baseline = True
    out = {}
    b = run_batch(sub, dist)
    out["batch"] = {k: b[k] for k in ("metric", "value", "unit", "ms_per_step", "plain_value", "plain_ms_per_step",
                                      "batched_no_graph_ms_per_step", "batched_over_plain", "gpu_launches",
                                      "clocks")}
    out["batch"]["steps"], out["batch"]["warmup"] = sub.steps, sub.warmup
    out["batch"]["workload"] = b["config"]["workload"]
    a = run_adjoint(sub, dist)
    out["adjoint"] = {k: a[k] for k in ("metric", "value", "unit", "ms_per_step", "forward_record_ms", "backward_ms",
                                        "plain_forward_ms", "backward_over_plain_forward", "gpu_launches", "clocks")}
    out["adjoint"]["steps"], out["adjoint"]["warmup"] = sub.steps, sub.warmup
    out["adjoint"]["workload"] = a["config"]["workload"]
    out["batch_over_plain"] = b["batched_over_plain"]
    out["adjoint_over_forward"] = a["value"]
    return out


def main():
    args = parse()
    dist = Dist(args.gpus)
    try:
        if args.workload == "large":
            line = run_large(args, dist) if args.impl == "ours" else \
                {"impl": "reference", "unavailable": "the large workload is measured on the GPU path only"}
        elif args.workload == "batch":
            line = run_batch(args, dist) if args.impl == "ours" else \
                {"impl": "reference", "unavailable": "the reference has no batched multi-scene form"}
        elif args.workload == "build":
            line = run_build(args, dist) if args.impl == "ours" else \
                {"impl": "reference", "unavailable": "the reference builds its BVHs with three-mesh-bvh in JS"}
        elif args.workload == "gather":
            line = run_gather(args, dist) if args.impl == "ours" else \
                {"impl": "reference", "unavailable": "the reference's gather is a WebGPU fragment shader"}
        elif args.workload == "adjoint":
            line = run_adjoint(args, dist) if args.impl == "ours" else \
                {"impl": "reference", "unavailable": "the reference has no adjoint of the probe update"}
        else:
            line = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
            if args.impl == "ours" and dist.world == 1 and not args.no_aux:
                line.update(aux_measurements(args, dist))
        if dist.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
