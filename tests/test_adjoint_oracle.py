"""The oracle's FP64 adjoint (oracle/orc_adjoint.hpp) on the CPU, no GPU.

Pins the hand-written reverse pass against central differences of the
oracle's own forward (the restated trace shading, blend and upload) on a small
room-and-spheres problem: 27 probes, 32 rays, 2 feedback solves, 6 materials,
5 point lights. With exact (unrounded) feedback the forward is smooth away
from its selects, so h = 1e-3 central differences agree with the adjoint to
O(h^2). Also checks that the adjoint's forward is the oracle's plain solve.
"""
import ctypes as C

import numpy as np
import pytest

from speedball_b200 import _abi
from speedball_b200 import scene as sc
from speedball_b200 import synth

H = 1e-3          # central-difference step (absolute, on albedo / emissive / light scale)
SOLVES = 2


@pytest.fixture(scope="module")
def problem(orc):
    s = synth.room_spheres(3, n_materials=6, n_point=5, n_dir=0)
    pool = sc.build_pool(s)
    mats, *_ = orc.compute_tail(pool)
    keep = []
    S = orc.scene_struct(pool, mats, keep=keep)
    g = dict(gridMin=(1.0, 1.0, 1.0), gridSize=(8.0, 8.0, 8.0), res=(3, 3, 3), rays=32)
    g["maxDist"] = float(np.linalg.norm(g["gridSize"]))
    g["cellMin"] = 4.0
    G = orc.grid_struct(g)
    recs = np.asarray(s.lights, np.float32).reshape(-1, 17)
    arena = orc.light_arena(recs, False, g)
    p = _abi.default_params()
    p.hysteresis = 0.97
    prm = p.to_array()
    probes, N = 27, 32
    n = probes * N
    irr, depth, atlas, datl = orc.new_state(g)
    io = orc.OrcSolveIO()
    tri, inst = np.zeros(n, np.int32), np.zeros(n, np.int32)
    blocked, facing = np.zeros(n, np.uint64), np.zeros(n, np.int32)
    io.hitTri, io.hitInst, io.blocked, io.hitFacing = orc._p(tri), orc._p(inst), orc._p(blocked), orc._p(facing)
    orc.solve(S, arena, recs.shape[0], False, G, G, prm, 0, probes, irr, depth, atlas, datl, io=io)
    word = np.where(tri >= 0, (inst.astype(np.uint32) | (facing.astype(np.uint32) << np.uint32(31))),
                    np.uint32(0xFFFFFFFF)).view(np.int32)
    mc = 6
    m = mats[: mc * 28].reshape(mc, 28).astype(np.float64)
    return dict(S=S, keep=keep, g=g, G=G, arena=arena, lights=recs.shape[0], prm=prm, tri=tri, word=word,
                blocked=blocked, mc=mc, albedo=m[:, 0:3].reshape(-1).copy(), emissive=m[:, 7:10].reshape(-1).copy(),
                mats=mats, pool=pool, recs=recs)


def _run(orc, P, albedo, emissive, scale, target=None, round_atlas=False, grad=True):
    return orc.adjoint(P["S"], P["arena"], P["lights"], False, P["G"], P["prm"], P["tri"], P["word"], P["blocked"],
                       SOLVES, albedo, emissive, scale, target=target, round_atlas=round_atlas, grad=grad)


def test_adjoint_forward_is_the_oracle_solve(orc, problem):
    """Two replayed solves through the adjoint's forward (rounded feedback)
    give the same upload output as two plain oracle solves."""
    P = problem
    g = P["g"]
    irr, depth, atlas, datl = orc.new_state(g)
    pre = np.zeros(27 * 36 * 3)
    for _ in range(SOLVES):
        io = orc.OrcSolveIO()
        io.replayTri, io.replayInst, io.replayBlocked = orc._p(P["tri"]), orc._p(P["word"]), orc._p(P["blocked"])
        io.preRound = orc._p(pre)
        orc.solve(P["S"], P["arena"], P["lights"], False, P["G"], P["G"], P["prm"], 0, 27, irr, depth, atlas, datl,
                  io=io)
    _, E, _ = _run(orc, P, P["albedo"], P["emissive"], np.ones(P["lights"]), round_atlas=True, grad=False)
    assert np.allclose(E, pre, rtol=1e-12, atol=1e-14)


def test_adjoint_matches_central_differences(orc, problem):
    P = problem
    rng = np.random.default_rng(11)
    mc, lc = P["mc"], P["lights"]
    albedo = P["albedo"]
    emissive = rng.uniform(0.0, 0.2, mc * 3)
    scale = np.ones(lc)
    # target: the forward with perturbed albedo and light intensity
    _, Et, _ = _run(orc, P, albedo * rng.uniform(0.8, 1.2, albedo.size), emissive, rng.uniform(0.5, 2.0, lc),
                    grad=False)
    loss, E, grad = _run(orc, P, albedo, emissive, scale, target=Et)
    assert loss > 0.0 and grad.shape == (6 * mc + lc,)
    theta = np.concatenate([albedo, emissive, scale])
    fd = np.zeros_like(theta)
    for j in range(theta.size):
        lo, hi = theta.copy(), theta.copy()
        lo[j] -= H
        hi[j] += H
        lp = _run(orc, P, hi[:3 * mc], hi[3 * mc:6 * mc], hi[6 * mc:], target=Et, grad=False)[0]
        lm = _run(orc, P, lo[:3 * mc], lo[3 * mc:6 * mc], lo[6 * mc:], target=Et, grad=False)[0]
        fd[j] = (lp - lm) / (2 * H)
    scale_g = np.abs(grad).max()
    err = np.abs(fd - grad)
    assert (err <= 1e-5 * scale_g + 1e-4 * np.abs(grad)).all(), (err.max(), scale_g, np.argmax(err))
    # every parameter family carries signal
    assert np.abs(grad[:3 * mc]).max() > 0 and np.abs(grad[3 * mc:6 * mc]).max() > 0
    assert np.abs(grad[6 * mc:]).max() > 0
