"""GPU: gdn_cuda_error_l2_noalloc, the allocation-free variant of the L2
error norm, for callers that cannot call cudaMalloc (hosts whose device memory
belongs to another allocator or to a fixed budget set at start-up).  Its
inputs are device buffers the caller owns (allocated here by the test, not by
the library); its result must equal the handle-based gdn_cuda_error_l2 on the
same state, on two calls in a row: on a mesh of one partial-sum block
(1,296 elements) and on one of six blocks whose last block is partly filled
(10,368 elements = 5 x 2,048 + 128).

Kept in its own file, collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn

pytestmark = pytest.mark.gpu

RTOL = 1e-10  # the tolerance the other error-norm tests use


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("n", [6, 12])
def test_error_l2_noalloc_matches_error_l2_twice(n):
    import torch
    coords, e2n = kuhn.kuhn_cube(n, 0.1, seed=4)
    mesh = capi.mesh_build(coords, e2n)
    ne = mesh.nbelems
    k = np.array([0.3, -0.4, 0.5])
    k /= np.linalg.norm(k)
    p = np.cross(k, [1.0, 0.0, 0.0])
    p /= np.linalg.norm(p)
    data = capi.plane_data(khat=k, kmag=3 * np.pi, pol=p)
    s = capi.Solver(mesh, capi.SCHEME_RK3, data, 0.3 * mesh.hmin())
    s.init()
    s.advance(6)
    expected = s.error_l2()
    wn = s.get_state()
    t = s.t
    wpg = np.ascontiguousarray(capi.tables_as_numpy(s.tables)["wpg"])
    s.close()

    # caller-owned device inputs
    xyz = mesh.node.reshape(-1, 3)[mesh.elem2qnode[: 10 * ne]]
    pv = mesh.node.reshape(-1, 3)[mesh.elem2qnode[: 10 * ne].reshape(ne, 10)[:, :4]]
    det = np.einsum("ij,ij->i", pv[:, 1] - pv[:, 0], np.cross(pv[:, 2] - pv[:, 0], pv[:, 3] - pv[:, 0]))
    w_d, x_d, d_d = _dev(torch, wn[: 60 * ne]), _dev(torch, xyz), _dev(torch, det)
    stream = torch.cuda.current_stream().cuda_stream
    L = capi.lib()
    got = []
    for _ in range(2):
        err = C.c_double(-1.0)
        capi.check(L.gdn_cuda_error_l2_noalloc(w_d.data_ptr(), x_d.data_ptr(), d_d.data_ptr(), ne,
                                               wpg.ctypes.data_as(C.POINTER(C.c_double)),
                                               C.byref(data), t, stream, C.byref(err)))
        got.append(err.value)
    for g in got:
        assert abs(g - expected) <= RTOL * expected, (g, expected)
    assert got[0] == got[1]


def test_error_l2_noalloc_rejects_oversize_mesh():
    import torch
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    wpg = np.ones(10)
    err = C.c_double()
    L = capi.lib()
    rc = L.gdn_cuda_error_l2_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 8388609,
                                     wpg.ctypes.data_as(C.POINTER(C.c_double)),
                                     C.byref(capi.plane_data()), 0.0, None, C.byref(err))
    assert rc == capi.ERR_INVALID
    assert b"8388608" in L.gdn_cuda_last_error()
