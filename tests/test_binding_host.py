"""The compiled binding (integration/dg_cuda.c in oracle/_ref/libgdon3d_ref_bound.so)
without a GPU: it exports what integration/dg_cuda.h declares, a simulation
that is not attached runs the reference's own dg_solve (renamed dg_solve_host)
bit for bit, and the reference-mesh fixtures written back as msh22 files read
as the reference read the originals."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gdon3d_b200 import kuhn
from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_meshes.npz")

needs_bound = pytest.mark.skipif(not ref.available("bound"),
                                 reason="oracle/_ref/libgdon3d_ref_bound.so not built")


@needs_bound
def test_bound_library_exports_the_binding():
    with open(os.path.join(ROOT, "integration", "dg_cuda.h")) as f:
        hdr = f.read()
    declared = set(re.findall(r"\b(dg_(?:cuda_[a-z_]+|solve_host))\s*\(", hdr)) | {"dg_solve"}
    assert {"dg_cuda_attach", "dg_cuda_detach", "dg_cuda_route_all", "dg_solve_host"} <= declared
    L = ref.lib("bound")
    for name in declared:
        assert hasattr(L, name), name


def test_fixture_meshes_round_trip_through_the_reference_reader(tmp_path):
    g = np.load(GOLDEN)
    for name in ("t4_cube_8", "t4_cube_16", "t4_cube_8_torus_128"):
        p = str(tmp_path / (name + ".msh"))
        kuhn.write_msh22(p, g[name + "_coords"], g[name + "_elem2node"])
        c, e = ref.msh_read_raw(p)
        assert np.array_equal(c, g[name + "_coords"])
        assert np.array_equal(e, g[name + "_elem2node"])


@needs_bound
@pytest.mark.parametrize("scheme,steps", [(ref.SCHEME_RK3, 5), (ref.SCHEME_D3Q4, 3)])
def test_unattached_dg_solve_is_the_reference_bit_for_bit(tmp_path, scheme, steps):
    g = np.load(GOLDEN)
    p = str(tmp_path / "t4_cube_8.msh")
    kuhn.write_msh22(p, g["t4_cube_8_coords"], g["t4_cube_8_elem2node"])
    d = ref.make_data(kind=ref.DATA_EXAMPLE_COS)
    dt = 0.032 / 9
    a = ref.RefMesh(path=p, variant="zero").run(scheme, d, dt, steps)
    b = ref.RefMesh(path=p, variant="bound").run(scheme, d, dt, steps)
    assert np.array_equal(a["wn"], b["wn"])
    assert a["t"] == b["t"]


@needs_bound
def test_binding_status_of_an_unattached_simulation_is_ok():
    L = ref.lib("bound")
    L.dg_cuda_status.restype = C.c_int
    L.dg_cuda_attached.restype = C.c_int
    dummy = C.create_string_buffer(256)
    assert L.dg_cuda_attached(dummy) == 0
    assert L.dg_cuda_status(dummy) == 0


@needs_bound
def test_unrouted_convergence_driver_is_the_reference(tmp_path):
    """The reference's utils_l2_time_convergence in the bound library, nothing routed, prints
    what the unmodified library prints."""
    g = np.load(GOLDEN)
    p = str(tmp_path / "t4_cube_8.msh")
    kuhn.write_msh22(p, g["t4_cube_8_coords"], g["t4_cube_8_elem2node"])
    dt = 0.3 * ref.RefMesh(path=p).hmin()
    d = ref.make_data(kind=ref.DATA_EXAMPLE_COS)
    a = ref.time_convergence(p, ref.SCHEME_RK3, d, dt, 12 * dt, 2, variant="zero")
    b = ref.time_convergence(p, ref.SCHEME_RK3, d, dt, 12 * dt, 2, variant="bound")
    assert len(a) == 2 and [r["iter"] for r in a] == [11, 22]
    assert [(r["dt"], r["iter"], r["error"]) for r in a] == [(r["dt"], r["iter"], r["error"]) for r in b]
