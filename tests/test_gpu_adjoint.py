"""The differentiated probe update on the GPU (sb_forward_record / sb_backward)
on the room-and-spheres scene with 64 materials and 32 point lights: 512
probes, 64 rays, 2 feedback solves, 416 parameters (64 x 3 albedo, 64 x 3
emissive, 32 light intensities). The target is the forward with albedo x
U[0.8, 1.2] and light intensity x U[0.5, 2].

Checked against the oracle's FP64 adjoint replaying the GPU's own hit records
and shadow bits (the same straight-through treatment of the RGBA16F feedback),
and against central differences (h = 1e-3) of the GPU forward itself.
"""
import json
import os

import numpy as np
import pytest

from speedball_b200 import _abi, synth
from speedball_b200.adjoint import GIAdjoint

from gpu_util import OracleMirror, gpu_records, make_field

pytestmark = pytest.mark.gpu

H = 1e-3
# GPU (FP32) gradient vs the FP64 adjoint: 1e-3 relative, with an absolute
# floor of 1e-5 of the largest gradient for near-zero components.
ADJ_REL, ADJ_FLOOR = 1e-3, 1e-5


@pytest.fixture(scope="module")
def diff_setup():
    s = synth.room_spheres(0, n_materials=64, n_point=32, n_dir=0)
    f = make_field(s)
    adj = GIAdjoint(f, solves=2)
    assert adj.materialCount == 64 and adj.lightCount == 32
    rng = np.random.default_rng(7)
    base = adj.parameters()
    adj.setParameters(albedo=base["albedo"] * rng.uniform(0.8, 1.2, (64, 3)), lightScale=rng.uniform(0.5, 2.0, 32))
    target = adj.forward()
    adj.setParameters(albedo=base["albedo"], lightScale=np.ones(32))
    loss = adj.forward(target)
    E = adj.readE()
    grads = adj.backward()
    yield dict(field=f, adj=adj, target=target, loss=loss, E=E, grads=grads, base=base)
    f.dispose()


def _flat(g):
    return np.concatenate([g["albedo"].reshape(-1), g["emissive"].reshape(-1), g["lightScale"].reshape(-1)])


def _report(name, data):
    out = os.environ.get("SB_ADJOINT_REPORT")
    if out:
        os.makedirs(os.path.dirname(out) or ".", exist_ok=True)
        rep = json.load(open(out)) if os.path.exists(out) else {}
        rep[name] = data
        json.dump(rep, open(out, "w"), indent=1)


def test_loss_is_sum_of_squares_of_E(diff_setup):
    d = diff_setup
    E, T = d["E"].astype(np.float64), d["target"].astype(np.float64)
    ref = float(((E - T) ** 2).sum())
    assert abs(d["loss"] - ref) <= 1e-9 * max(ref, 1e-30)
    assert d["loss"] > 0


def test_backward_needs_a_current_tape(diff_setup):
    d = diff_setup
    adj = d["adj"]
    adj.setParameters(lightScale=np.full(32, 1.0 + 1e-3))
    with pytest.raises(_abi.SbError):
        adj.backward()
    adj.setParameters(lightScale=np.ones(32))
    adj.forward(d["target"])  # restore the recorded tape at the base point


def test_gradients_match_fp64_adjoint(diff_setup, orc):
    d = diff_setup
    f, adj = d["field"], d["adj"]
    adj.forward(d["target"])
    g_gpu = _flat(adj.backward())
    mirror = OracleMirror(f)
    n = adj.probes * f.getRays()
    rec = gpu_records(f, n)
    base = d["base"]
    loss, E, g_orc = orc.adjoint(mirror.scene, mirror.arena, mirror.light_count, mirror.clustered, mirror.grid,
                                 mirror.params(), rec["tri"], rec["inst_word"], rec["blocked"], 2,
                                 base["albedo"].astype(np.float32).astype(np.float64).reshape(-1),
                                 base["emissive"].reshape(-1), np.ones(32),
                                 target=d["target"].astype(np.float64).reshape(-1), round_atlas=True)
    eg = d["E"].astype(np.float64).reshape(-1)
    e_rel = np.abs(eg - E) / np.maximum(np.abs(E), 1e-3 * np.abs(E).max())
    err = np.abs(g_gpu - g_orc)
    scale = np.abs(g_orc).max()
    rel = err / np.maximum(np.abs(g_orc), ADJ_FLOOR / ADJ_REL * scale)
    _report("fp64_adjoint", dict(loss_gpu=d["loss"], loss_fp64=loss, E_rel_max=float(e_rel.max()),
                                 grad_rel_max=float(rel.max()), grad_rel_median=float(np.median(rel)),
                                 grad_abs_scale=float(scale),
                                 per_family_rel_max=[float(rel[:192].max()), float(rel[192:384].max()),
                                                     float(rel[384:].max())]))
    assert e_rel.max() <= 1e-3
    assert abs(d["loss"] - loss) <= 1e-3 * loss
    assert (err <= ADJ_REL * np.abs(g_orc) + ADJ_FLOOR * scale).all(), (rel.max(), int(np.argmax(rel)))


def test_gradients_match_central_differences(diff_setup):
    d = diff_setup
    adj, target = d["adj"], d["target"]
    base = d["base"]
    adj.forward(target)
    g = _flat(adj.backward())
    theta = np.concatenate([base["albedo"].reshape(-1), base["emissive"].reshape(-1), np.ones(32)])
    fd = np.zeros_like(theta)

    def set_theta(t):
        adj.setParameters(albedo=t[:192].reshape(64, 3), emissive=t[192:384].reshape(64, 3), lightScale=t[384:])

    for j in range(theta.size):
        hi, lo = theta.copy(), theta.copy()
        hi[j] += H
        lo[j] -= H
        # the step the float32 records actually took
        step = float(np.float32(hi[j]) - np.float32(lo[j])) if j < 384 else 2 * H
        set_theta(hi)
        lp = adj.forward(target)
        set_theta(lo)
        lm = adj.forward(target)
        fd[j] = (lp - lm) / step
    set_theta(theta)
    scale = np.abs(g).max()
    err = np.abs(fd - g)
    rel = err / np.maximum(np.abs(g), 1e-2 * scale)
    norm_rel = float(np.linalg.norm(fd - g) / np.linalg.norm(g))
    fam = [slice(0, 192), slice(192, 384), slice(384, 416)]
    _report("central_differences", dict(h=H, norm_rel=norm_rel, rel_max=float(rel.max()),
                                        rel_median=float(np.median(rel)),
                                        family_norm_rel=[float(np.linalg.norm(fd[s] - g[s]) / np.linalg.norm(g[s]))
                                                         for s in fam],
                                        worst=[int(i) for i in np.argsort(-rel)[:8]],
                                        worst_g=[float(g[i]) for i in np.argsort(-rel)[:8]],
                                        worst_fd=[float(fd[i]) for i in np.argsort(-rel)[:8]]))
    # 1e-3 relative as a vector norm; per component 1e-3 relative with an
    # absolute floor of 1e-4 of the largest gradient (the FP32 forward and the
    # binary16 feedback make differences of small components noisy)
    assert norm_rel <= 1e-3, norm_rel
    assert (err <= 1e-3 * np.abs(g) + 1e-4 * scale).all(), (rel.max(), int(np.argmax(rel)))
