"""giEmitter lights (emissive spheres): the emitter visibility kernel and the
blend's virtual rays (gi_probes.js:2216-2310) against the oracle.

The room scene gets one emissive icosphere (a sphere emitter with its bounding
radius) and two point-like emitters of radius 0, whose visibility ray ends at
the centre whatever the hash (so every sample is a plain any-hit query). Over
montecarlo ticks (a new emitter seed each tick) every solve is checked:
  * the point emitters' visibility samples equal the FP64 oracle's on every
    updated probe; the sphere emitter's disk point comes from a float32 sin
    hash whose last ulp differs between libraries, so its samples must agree
    on at least 97% of probes;
  * the oracle, given the GPU's visibility history, reproduces every
    irradiance and depth texel within 1e-3 (the virtual rays' arithmetic);
  * hit IDs ray by ray as in the other parity tests.
Batched solves and the adjoint refuse emitters (SB_ERR_UNSUPPORTED).
"""
import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu


def test_emitter_visibility_and_virtual_rays_match_oracle():
    s = synth.add_emitters(synth.room_spheres(0))
    f = gu.make_field(s)
    try:
        f.setJitterMode("montecarlo")
        mirror = gu.OracleMirror(f)
        assert mirror.emitters == (5, 3)
        sched = orc.Schedule(f._probeTotal, f.getRays(), f._rayBudget, f._maxProbesPerTick, True, False)
        seeds = []
        for k in range(4):
            frame = f.tick(nowMs=100.0 + 16.0 * k)
            f.synchronize()
            want = sched.tick(100.0 + 16.0 * k)
            assert (frame["probeOffset"], frame["updatedCount"]) == (want["probeOffset"], want["updatedCount"])
            prm = f._params.to_array()
            seeds.append(float(prm[orc.ORC_PARAM_NAMES.index("emitterVisSeed")]))
            r = gu.solve_parity(f, mirror, frame, prm)
            agree = r["emitter_sample_agreement"]
            print(k, agree, r["irr_err"])
            assert agree[1] == 1.0 and agree[2] == 1.0, agree
            assert agree[0] >= 0.97, agree
        assert len(set(seeds)) == 4
        vis = gu.read(f, "EMITTER_VIS", f._probeTotal * 16, np.float32).reshape(-1, 16)
        assert 0.0 < vis[:, :3].mean() < 1.0 and np.all(vis[:, 3:] == 0.0)
    finally:
        f.dispose()


def test_batched_solves_and_adjoint_refuse_emitters():
    s = synth.add_emitters(synth.room_spheres(0))
    f = gu.make_field(s)
    try:
        items = (_abi.sb_solve_item * 1)()
        items[0].ctx = f.ctx
        items[0].cascade = 0
        items[0].probeOffset = 0
        items[0].updatedCount = f._probeTotal
        assert f._lib.sb_solve_batch(items, 1) == _abi.SB_ERR_UNSUPPORTED
        loss = _abi.C.c_double(0.0)
        assert f._lib.sb_forward_record(f.ctx, 0, 1, None, _abi.C.byref(loss)) == _abi.SB_ERR_UNSUPPORTED
        f.tick()
        f.synchronize()
    finally:
        f.dispose()
