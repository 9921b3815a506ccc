"""Receiver gather (sb_gather_irradiance) against the oracle's FP64
restatement of GiProbeNode's gather (gi_probes.js:530-657, 816-850, 884-928),
on the atlases of a real solve sequence read back from the GPU.

Samples are surface points and normals spread through the probe grid. Each
irradiance component must agree within 1e-3 relative (floor 1e-3 of the
largest magnitude), the texel bar of the update. Samples within 1e-4 cell of a
cage-selection boundary, or within 1e-4 relative of the Chebyshev select, are
discontinuities where FP32 and FP64 may pick different sides; they are counted
and must be rare, and are not compared.
"""
import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 200_000


@pytest.fixture(scope="module")
def field():
    s = synth.room_spheres(0)
    f = gu.make_field(s)
    g = s.meta["grid"]
    # a fine box: the half-extent box around the centre, 8^3 probes
    gmin = np.asarray(g["gridMin"], np.float64)
    gsz = np.asarray(g["gridSize"], np.float64)
    f.configureCascade(1, (gmin + gsz * 0.25).tolist(), (gsz * 0.5).tolist(), (8, 8, 8))
    for _ in range(4):
        fr = f.beginTick()
        _abi.check(f._lib.sb_solve(f.ctx, 0, fr["probeOffset"], fr["updatedCount"]), f.ctx)
        _abi.check(f._lib.sb_solve(f.ctx, 1, 0, f.cascadeProbes(1)), f.ctx)
        f.endTick(fr)
    f.synchronize()
    yield s, f
    f.dispose()


def _samples(g: dict, n: int, seed: int):
    rng = np.random.default_rng(seed)
    lo = np.asarray(g["gridMin"], np.float64) - 0.1
    hi = lo + np.asarray(g["gridSize"], np.float64) + 0.2
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, (n, 3))
    nv = rng.normal(size=(n, 3))
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    nd = nv + rng.normal(0, 0.3, (n, 3))
    nd /= np.linalg.norm(nd, axis=1, keepdims=True)
    a = np.zeros((n, 4), np.float32); a[:, :3] = nv
    b = np.zeros((n, 4), np.float32); b[:, :3] = nd
    return pos, a, b


def _gpu_gather(f, prm, pos, nv, nd):
    dev = torch.device("cuda", 0)
    tp, tn, td = (torch.from_numpy(x).to(dev) for x in (pos, nv, nd))
    out = torch.zeros((pos.shape[0], 4), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    _abi.check(f._lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), tp.data_ptr(), tn.data_ptr(), td.data_ptr(),
                                           pos.shape[0], out.data_ptr()), f.ctx)
    f.synchronize()
    return out.cpu().numpy()


def _atlases(f, ci):
    g = f.grid if ci == 0 else f._extraCascades[ci]
    r = [g.res[a] for a in range(3)]
    W, H = r[0] * 8, r[1] * r[2] * 8
    a = gu.read(f, "IRRADIANCE_ATLAS", W * H * 4, np.uint16, ci)
    d = gu.read(f, "DEPTH_ATLAS", W * H * 4, np.uint16, ci)
    return orc.grid_struct(gu.grid_dict(g)), a, d


CASES = {
    "defaults": dict(),
    "chebyshev_dual_detail": dict(chebyStrength=1.0, chebyBias0=0.05, dualDetail=1.0, detailStrength=0.5,
                                  normalBias0=0.05),
    "two_cascades": dict(cascades=2.0, chebyStrength=1.0, chebyBias0=0.02, chebyBias1=0.01, borderBand=0.2),
}


@pytest.mark.parametrize("case", list(CASES))
def test_gather_matches_oracle(field, case):
    s, f = field
    kw = CASES[case]
    prm = _abi.sb_gather_params()
    f._lib.sb_gather_params_defaults(_abi.C.byref(prm))
    prm.normalBias[0] = kw.get("normalBias0", 0.04)
    prm.chebyBias[0] = kw.get("chebyBias0", 0.0)
    prm.chebyBias[1] = kw.get("chebyBias1", 0.0)
    prm.chebyStrength = kw.get("chebyStrength", 0.0)
    prm.detailStrength = kw.get("detailStrength", 1.0)
    prm.borderBand = kw.get("borderBand", 0.15)
    prm.cascades = int(kw.get("cascades", 1))
    prm.dualDetail = int(kw.get("dualDetail", 0))
    pos, nv, nd = _samples(s.meta["grid"], N, 5)
    got = _gpu_gather(f, prm, pos, nv, nd)
    G0, a0, d0 = _atlases(f, 0)
    G1, a1, d1 = _atlases(f, 1)
    oprm = orc.gather_params(**kw)
    want, near = orc.gather(G0, a0, d0, oprm, pos, nv, nd, G1 if prm.cascades == 2 else None,
                            a1 if prm.cascades == 2 else None, d1 if prm.cascades == 2 else None)
    edge = near < 1e-4
    assert edge.mean() < 2e-3, edge.mean()
    err = gu.texel_rel_err(got[~edge, :3].reshape(-1).astype(np.float64), want[~edge].reshape(-1))
    print(case, "max rel err", err.max(), "discontinuity samples", int(edge.sum()))
    assert err.max() <= gu.TEXEL_REL, (case, err.max(), int((err > gu.TEXEL_REL).sum()))
    assert np.all(got[:, 3] == 1.0)
    assert want.max() > 0.01  # the field is lit


def test_gather_rejects_bad_arguments(field):
    s, f = field
    prm = _abi.sb_gather_params()
    f._lib.sb_gather_params_defaults(_abi.C.byref(prm))
    dev = torch.device("cuda", 0)
    buf = torch.zeros((65, 4), dtype=torch.float32, device=dev)
    p = buf.data_ptr()
    lib = f._lib
    assert lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), p + 4, p, p, 8, p) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), None, p, p, 8, p) == _abi.SB_ERR_INVALID_ARG
    prm.cascades = 3
    assert lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), p, p, p, 8, p) == _abi.SB_ERR_INVALID_ARG
    prm.cascades = 2
    prm.dualDetail = 1
    assert lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), p, p, p, 8, p) == _abi.SB_ERR_INVALID_ARG
    prm.cascades = 1
    prm.dualDetail = 0
    assert lib.sb_gather_irradiance(f.ctx, _abi.C.byref(prm), p, p, p, 0, p) == _abi.SB_OK
