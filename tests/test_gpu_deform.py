"""The deform lane from attribute arrays (sb_update_deform_xyz, updateDeforms,
spectral_scene.js:1831-1927): positions and normals replace the first six
floats of the mesh's pooled vertices, uv keeps its build-time value, and the
BLAS refit that follows equals the oracle's refit of the same vertices bit for
bit. Without normals the build-time normals stay too. Bad ranges are refused."""
import numpy as np
import pytest

import orc
from speedball_b200 import _abi, synth

import gpu_util as gu

pytestmark = pytest.mark.gpu


def test_deform_from_attribute_arrays_matches_oracle():
    s = synth.room_spheres(0)
    f = gu.make_field(s)
    try:
        pool = f.pool
        mesh = int(np.argmax(pool.vert_count))
        vb, vc = int(pool.vert_base[mesh]), int(pool.vert_count[mesh])
        root, end = int(pool.blas_root[mesh]), int(pool.blas_end[mesh])
        before = gu.read(f, "VERTEX_DATA", pool.vertexData.size, np.float32).reshape(-1, 8)
        nodes = gu.read(f, "BVH_NODES", pool.bvhNodes.size, np.uint32).reshape(-1, 8)
        rng = np.random.default_rng(3)
        pos = (before[vb:vb + vc, 0:3] + rng.normal(0, 0.05, (vc, 3))).astype(np.float32)
        nrm = rng.normal(0, 1, (vc, 3)).astype(np.float32)
        for normals in (nrm, None):
            _abi.check(f._lib.sb_update_deform_xyz(f.ctx, vb, vc, _abi.ptr(pos),
                                                   None if normals is None else _abi.ptr(normals), root, end), f.ctx)
            f.synchronize()
            after = gu.read(f, "VERTEX_DATA", pool.vertexData.size, np.float32).reshape(-1, 8)
            want = before.copy()
            want[vb:vb + vc, 0:3] = pos
            want[vb:vb + vc, 3:6] = nrm  # the first call's normals stay through the second
            assert np.array_equal(after, want)
            got_nodes = gu.read(f, "BVH_NODES", pool.bvhNodes.size, np.uint32).reshape(-1, 8)
            ref_nodes = nodes.copy()
            ref_vertex = np.ascontiguousarray(want.reshape(-1))
            assert orc.load().orc_refit_blas(orc._p(ref_nodes), ref_nodes.size, orc._p(pool.triIndex),
                                             pool.triIndex.size, orc._p(ref_vertex), ref_vertex.size, root, end) == 1
            assert np.array_equal(got_nodes, ref_nodes)
            pos = (pos + 0.01).astype(np.float32)
        # a range outside the pool and a null position array are refused before any work
        assert f._lib.sb_update_deform_xyz(f.ctx, vb, pool.vertexData.size, _abi.ptr(pos), None, root,
                                           end) == _abi.SB_ERR_INVALID_ARG
        assert f._lib.sb_update_deform_xyz(f.ctx, vb, vc, None, None, root, end) == _abi.SB_ERR_INVALID_ARG
    finally:
        f.dispose()
