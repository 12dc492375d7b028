"""gdn_cuda_mesh_build_gpu builds the connectivity arrays of the host builder
(the reference's mesh_build_connectivity conventions) bit for bit."""
import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,jitter", [(1, 0.0), (3, 0.0), (5, 0.15), (17, 0.1)])
def test_mesh_build_gpu_equals_host(n, jitter):
    c, e = kuhn.kuhn_cube(n, jitter, seed=n)
    h = capi.mesh_build(c, e)
    g = capi.mesh_build(c, e, device=0)
    for name in ("face2elem", "fnode2enode", "boundaryface", "elem2qnode", "node"):
        assert np.array_equal(getattr(h, name), getattr(g, name)), name
    assert (h.nbelems, h.nbfaces, h.nboundaryfaces, h.nbqnodes) == (g.nbelems, g.nbfaces, g.nboundaryfaces,
                                                                     g.nbqnodes)


def test_mesh_build_gpu_rejects_bad_indices():
    c, e = kuhn.kuhn_cube(2)
    e = e.copy()
    e[0, 0] = 10 ** 6
    with pytest.raises(capi.GdnError) as ex:
        capi.mesh_build(c, e, device=0)
    assert ex.value.code == capi.ERR_MESH
