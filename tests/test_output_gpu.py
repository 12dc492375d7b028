"""gdn_cuda_save_xdmf: io_save_all's content (io_hdf5.c) as raw binary files
described by an XDMF file: connectivity, P2 nodes, and each node's state
components taken at its first element and first local node."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn

pytestmark = pytest.mark.gpu


def _expected(mesh, wn, m, kinetic, nb_v):
    ne, nq = mesh.nbelems, mesh.nbqnodes
    e2q = mesh.elem2qnode[: 10 * ne]
    owner = np.full(nq, -1, np.int64)
    for u in range(10 * ne):  # element order, first local node
        if owner[e2q[u]] < 0:
            owner[e2q[u]] = u
    neq = 10 * ne + 6 * mesh.nboundaryfaces
    out = np.zeros((m, nq))
    for im in range(m):
        if kinetic:
            out[im] = wn[im * neq + owner]
        else:
            out[im] = wn[owner * 6 + im]
    return out


@pytest.mark.parametrize("scheme,nb_v", [(capi.SCHEME_RK3, 0), (capi.SCHEME_KINETIC, 4)])
def test_save_xdmf_writes_the_reference_content(tmp_path, scheme, nb_v):
    c, e = kuhn.kuhn_cube(3, 0.1, seed=5)
    mesh = capi.mesh_build(c, e)
    mult = 1 if scheme == capi.SCHEME_RK3 else 10
    s = capi.Solver(mesh, scheme, capi.cavity_data(), mult * 0.3 * mesh.hmin(), nb_v=nb_v or 4)
    wn, t, _ = s.solve(3)
    base = str(tmp_path / "run")
    s.save_xdmf(base, 3)
    m = 6 if scheme == capi.SCHEME_RK3 else 24
    s.close()
    ne, nq = mesh.nbelems, mesh.nbqnodes
    conn = np.fromfile(base + "_mesh_conn.bin", dtype="<i4").reshape(ne, 10)
    nodes = np.fromfile(base + "_mesh_nodes.bin", dtype="<f8").reshape(nq, 3)
    data = np.fromfile(base + "_data_0003.bin", dtype="<f8").reshape(m, nq)
    assert np.array_equal(conn.ravel(), mesh.elem2qnode[: 10 * ne])
    assert np.array_equal(nodes.ravel(), mesh.node)
    assert np.array_equal(data, _expected(mesh, wn, m, scheme == capi.SCHEME_KINETIC, 4))
    root = ET.parse(base + "_simulation_0003.xmf").getroot()
    grid = root.find("Domain/Grid")
    assert grid.find("Topology").get("TopologyType") == "Tet_10"
    assert float(grid.find("Time").get("Value")) == pytest.approx(t, abs=1e-6)
    names = [a.get("Name") for a in grid.findall("Attribute")]
    if scheme == capi.SCHEME_RK3:
        assert names == ["w%d" % i for i in range(6)]
    else:
        assert names == ["f%d" % i for i in range(24)] + ["w%d" % i for i in range(6)]
    seeks = [int(d.get("Seek")) for d in grid.findall("Attribute/DataItem") if d.get("Seek") is not None]
    assert seeks[:m] == [im * nq * 8 for im in range(m)]
    assert os.path.basename(base) + "_data_0003.bin" in ET.tostring(grid).decode()


@pytest.mark.parametrize("scheme", [capi.SCHEME_RK3, capi.SCHEME_KINETIC])
def test_save_xdmf_of_a_batch_instance_equals_its_single_solve(tmp_path, scheme):
    """The files written for instance i of a batch handle (instance-local
    connectivity and nodes, its own state and time) are byte-identical to
    those of the same instance solved alone."""
    specs = [(2, 0.1, 1), (3, 0.0, 2), (2, 0.15, 3)]
    meshes, datas, dts = [], [], []
    for k, (n, jitter, seed) in enumerate(specs):
        c, e = kuhn.kuhn_cube(n, jitter, seed=seed)
        meshes.append(capi.mesh_build(c, e))
        datas.append(capi.plane_data(kmag=2 * np.pi * (1 + k)))
        dts.append((1 if scheme == capi.SCHEME_RK3 else 10) * 0.3 * meshes[-1].hmin())
    b = capi.BatchSolver(meshes, datas, dts, scheme=scheme, rk3_variant=1)
    b.solve(4)
    for i in (1, 2):
        b.save_xdmf(str(tmp_path / ("batch%d" % i)), 4, instance=i)
    b.close()
    for i in (1, 2):
        s = capi.Solver(meshes[i], scheme, datas[i], dts[i], rk3_variant=1)
        s.solve(4)
        s.save_xdmf(str(tmp_path / ("single%d" % i)), 4)
        s.close()
        for suffix in ("_mesh_conn.bin", "_mesh_nodes.bin", "_data_0004.bin"):
            a = (tmp_path / ("batch%d%s" % (i, suffix))).read_bytes()
            o = (tmp_path / ("single%d%s" % (i, suffix))).read_bytes()
            assert a == o, (i, suffix)
        xa = (tmp_path / ("batch%d_simulation_0004.xmf" % i)).read_text().replace("batch%d" % i, "X")
        xo = (tmp_path / ("single%d_simulation_0004.xmf" % i)).read_text().replace("single%d" % i, "X")
        assert xa == xo, i
