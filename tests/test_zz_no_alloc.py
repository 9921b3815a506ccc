"""sb_refit_blas_static: the BLAS refit that allocates nothing, checked against
sb_refit_blas (the context path) on the same node, triangle and vertex pools.
Node bounds are bit-exact on both paths, so the comparison is bit-exact too.
Collected last so it also runs after every other test in the same process."""
import ctypes as C

import numpy as np
import pytest

from speedball_b200 import _abi
from speedball_b200 import synth

MAX_NODES = 524288  # SB_REFIT_STATIC_MAX_NODES


def _call(lib, nodes_d, n_nodes, tri_d, n_tris, vert_d, n_verts, root, end, stream):
    msg = C.create_string_buffer(256)
    st = lib.sb_refit_blas_static(nodes_d, n_nodes, tri_d, n_tris, vert_d, n_verts, root, end, stream,
                                  msg, len(msg))
    return st, msg.value.decode()


def test_static_refit_rejects_oversize_range_before_device_work():
    lib = _abi.load()
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    st, msg = _call(lib, fake, MAX_NODES + 10, fake, 1, fake, 1, 0, MAX_NODES + 1, None)
    assert st == _abi.SB_ERR_INVALID_ARG and "maximum" in msg
    st, msg = _call(lib, None, 8, fake, 1, fake, 1, 0, 4, None)
    assert st == _abi.SB_ERR_INVALID_ARG
    st, msg = _call(lib, fake, 8, fake, 1, fake, 1, 4, 9, None)
    assert st == _abi.SB_ERR_LAYOUT_VIOLATION


@pytest.mark.gpu
def test_static_refit_matches_context_refit_on_consecutive_calls():
    import torch
    import gpu_util as gu

    s = synth.room_spheres(0)
    f = gu.make_field(s, record=False)
    try:
        pool = f.pool
        lib = f._lib
        dev = torch.device("cuda", 0)
        nodes_d = torch.from_numpy(pool.bvhNodes.reshape(-1).view(np.int32).copy()).to(dev)
        tri_d = torch.from_numpy(pool.triIndex.reshape(-1).view(np.int32).copy()).to(dev)
        vert_host = pool.vertexData.copy()
        vert_d = torch.from_numpy(vert_host.reshape(-1).copy()).to(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        n_nodes, n_tris, n_verts = pool.bvhNodes.shape[0], pool.triIndex.shape[0], pool.vertexData.shape[0]
        rng = np.random.default_rng(11)

        def deform_and_compare(m):
            vb, vc = int(pool.vert_base[m]), int(pool.vert_count[m])
            root, end = int(pool.blas_root[m]), int(pool.blas_end[m])
            vert_host[vb:vb + vc, 0:3] += rng.normal(0, 0.05, (vc, 3)).astype(np.float32)
            sl = np.ascontiguousarray(vert_host[vb:vb + vc])
            # context path: upload the slice, refit, read the pool back
            _abi.check(lib.sb_upload_range(f.ctx, _abi.BUF["VERTEX_DATA"], vb * 8, vc * 8, _abi.ptr(sl)), f.ctx)
            _abi.check(lib.sb_refit_blas(f.ctx, root, end), f.ctx)
            f.synchronize()
            want = gu.read(f, "BVH_NODES", pool.bvhNodes.size, np.uint32)
            # no-allocation path on the caller's own buffers
            vert_d[vb * 8:(vb + vc) * 8] = torch.from_numpy(sl.reshape(-1)).to(dev)
            st, msg = _call(lib, nodes_d.data_ptr(), n_nodes, tri_d.data_ptr(), n_tris, vert_d.data_ptr(),
                            n_verts, root, end, stream)
            assert st == _abi.SB_OK, msg
            got = nodes_d.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, want)
            before = pool.bvhNodes.reshape(-1)[root * 8:end * 8]
            assert not np.array_equal(got[root * 8:end * 8], before)  # the refit moved the bounds

        deform_and_compare(1)   # first call on the device: its device code and scratch address
        deform_and_compare(1)   # same range again: scratch from the last call is cleared
        # a range whose right child escapes it fails closed and leaves the pool usable
        r, e = int(pool.blas_root[3]), int(pool.blas_end[3])
        st, msg = _call(lib, nodes_d.data_ptr(), n_nodes, tri_d.data_ptr(), n_tris, vert_d.data_ptr(),
                        n_verts, r, e - 1, stream)
        assert st == _abi.SB_ERR_LAYOUT_VIOLATION, msg
        deform_and_compare(7)   # a different range after the failed call
    finally:
        f.dispose()


def _tiny_pool():
    """Three triangles of three vertices each; a root over two leaves (pre-order,
    left child at i + 1): node 0 interior, node 1 leaf of triangles 0-1, node 2
    leaf of triangle 2. Bounds start as a stale unit box."""
    rng = np.random.default_rng(5)
    vert = np.zeros((9, 8), np.float32)
    vert[:, 0:3] = rng.uniform(-2, 2, (9, 3))
    tri = np.arange(9, dtype=np.uint32)
    nodes = np.zeros((3, 8), np.uint32)
    stale = np.array([-1, -1, -1, 1, 1, 1], np.float32).view(np.uint32)
    for i in range(3):
        nodes[i, 0:6] = stale
    nodes[0, 6], nodes[0, 7] = 3, 0xFFFFFFFF
    nodes[1, 6], nodes[1, 7] = 2, (2 << 24) | 0
    nodes[2, 6], nodes[2, 7] = 3, (1 << 24) | 2
    return nodes, tri, vert


@pytest.mark.gpu
def test_static_refit_edge_pools():
    """The static path's own branches on tiny pools: an empty leaf keeps its
    stale bounds exactly as the oracle's refitFlatBlasRange restatement does;
    a leaf whose triangles lie past triCount, and a range holding a node no
    parent reaches, fail with SB_ERR_LAYOUT_VIOLATION and leave the nodes
    untouched."""
    import torch
    import orc

    lib = _abi.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def run(nodes, tri, vert, root, end):
        nd = torch.from_numpy(nodes.reshape(-1).view(np.int32).copy()).to(dev)
        td = torch.from_numpy(tri.view(np.int32).copy()).to(dev)
        vd = torch.from_numpy(vert.reshape(-1).copy()).to(dev)
        st, msg = _call(lib, nd.data_ptr(), nodes.shape[0], td.data_ptr(), tri.size // 3, vd.data_ptr(),
                        vert.shape[0], root, end, stream)
        torch.cuda.synchronize()
        return st, msg, nd.cpu().numpy().view(np.uint32).reshape(-1, 8)

    # an empty leaf (count 0): bit-equal to the oracle's refit of the same pool
    nodes, tri, vert = _tiny_pool()
    nodes[2, 7] = (0 << 24) | 2
    st, msg, got = run(nodes, tri, vert, 0, 3)
    want = nodes.copy()
    assert orc.load().orc_refit_blas(orc._p(want), want.size, orc._p(tri), tri.size, orc._p(vert), vert.size, 0, 3) == 1
    assert st == _abi.SB_OK, msg
    assert np.array_equal(got, want)
    assert np.array_equal(got[2, 0:6], nodes[2, 0:6])  # the empty leaf kept its stale box
    assert not np.array_equal(got[1, 0:6], nodes[1, 0:6])

    # a leaf whose triangles run past triCount
    nodes, tri, vert = _tiny_pool()
    nodes[2, 7] = (2 << 24) | 2  # triangles 2 and 3 of 3
    st, msg, got = run(nodes, tri, vert, 0, 3)
    assert st == _abi.SB_ERR_LAYOUT_VIOLATION, msg
    assert np.array_equal(got, nodes)

    # a node that no parent reaches: node 3 after the root's subtree, inside the range
    nodes, tri, vert = _tiny_pool()
    extra = nodes[2:3].copy()
    extra[0, 6] = 4
    nodes4 = np.concatenate([nodes, extra])
    st, msg, got = run(nodes4, tri, vert, 0, 4)
    assert st == _abi.SB_ERR_LAYOUT_VIOLATION, msg
    assert np.array_equal(got, nodes4)
