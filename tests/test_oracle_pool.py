"""The oracle's own scene pool (MeshBVH restatement + pool assembly) against
the library's host pool, and the reference arm's independence from the CUDA
library. CPU only."""
import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

from speedball_b200 import scene as sc
from speedball_b200 import synth

import orc

ROOT = Path(__file__).resolve().parents[1]


def _tail(pool):
    mats, order, live, aabb = orc.compute_tail(pool)
    keep = [pool]
    return orc.scene_struct(pool, mats, keep=keep), keep


def test_oracle_pool_layout_checks_pass_for_every_blas():
    s = synth.room_spheres(0)
    p = orc.OrcPool(s)
    assert p.triIndex.shape[0] == sum(m.indices.shape[0] for m in s.meshes)
    lib = orc.load()
    for m in range(len(s.meshes)):
        nodes = p.bvhNodes.copy()
        assert lib.orc_refit_blas(orc._p(nodes), nodes.size, orc._p(p.triIndex), p.triIndex.size,
                                  orc._p(p.vertexData), p.vertexData.size, int(p.blas_root[m]),
                                  int(p.blas_end[m])) == 1, m
        # leaves of at most 8 triangles cover every triangle of the mesh exactly once
        seg = p.bvhNodes[p.blas_root[m]:p.blas_end[m]]
        leaf = seg[seg[:, 7] != 0xFFFFFFFF, 7]
        cnt = leaf >> 24
        off = leaf & 0xFFFFFF
        assert cnt.max() <= 8 and cnt.min() >= 1
        covered = np.concatenate([np.arange(o, o + c) for o, c in zip(off, cnt)])
        assert np.array_equal(np.sort(covered), np.arange(covered.min(), covered.min() + covered.size))
    # every triangle keeps its material through the permutation
    src = np.concatenate([m.tri_material for m in s.meshes])
    assert np.array_equal(np.sort(p.triMaterial), np.sort(src))


def test_oracle_pool_gives_the_library_pool_hits():
    """Two different valid BVHs over the same triangles give the same closest
    hit on every ray except exactly equal t (the first visited wins a tie)."""
    s = synth.room_spheres(0)
    po = orc.OrcPool(s)
    pl = sc.build_pool(s)
    so, ko = _tail(po)
    sl, kl = _tail(pl)
    rng = np.random.default_rng(3)
    n = 20_000
    ro = rng.uniform(0.3, 9.7, (n, 3)).astype(np.float32)
    rd = rng.normal(size=(n, 3))
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    out = {}
    for key, S in (("orc", so), ("lib", sl)):
        t, tri, inst, t2 = np.zeros(n), np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n)
        orc.load().orc_closest(C.byref(S), orc._p(ro), orc._p(rd), n, 1, 0, orc._p(t), orc._p(tri), orc._p(inst),
                               orc._p(t2), orc.threads())
        out[key] = (t, tri, inst, t2)
    assert np.array_equal(out["orc"][0], out["lib"][0])  # the nearest t is the same number
    # triangle ids differ between the pools (BVH order): compare the source triangle
    def src_tri(pool, tri, inst):
        return np.where(tri >= 0, pool.triIndex[np.maximum(tri, 0)].sum(1), -1)
    same = src_tri(po, out["orc"][1], out["orc"][2]) == src_tri(pl, out["lib"][1], out["lib"][2])
    tie = out["orc"][3] == out["orc"][0]
    assert (~same & ~tie).sum() == 0
    assert (out["orc"][1] >= 0).mean() > 0.9


def test_reference_arm_does_not_load_the_cuda_library():
    code = (
        "import sys, json; sys.argv=['bench.py','--impl','reference','--steps','1','--warmup','1'];"
        f"sys.path.insert(0, {str(ROOT)!r}); import bench; bench.main();"
        "maps=open('/proc/self/maps').read();"
        "print('LOADED', 'libspeedball_cuda' in maps, 'liborc' in maps)"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "LOADED False True" in r.stdout, r.stdout[-2000:]
