"""HP-1 parity on the GPU: the FP64 RK3 path against the reference's own C code
(oracle/_ref, compiled from the reference sources) on the same mesh, data and
dt.  Bar: relative L2 of the whole state vector <= 1e-12 (FP64 path), FP32
path within its stated tolerance."""
import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn
from oracle import ref

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12


def _run_pair(n, jitter, steps, data_kw, seed=3, precision=capi.FP64):
    c, e = kuhn.kuhn_cube(n, jitter, seed=seed)
    mesh = capi.mesh_build(c, e)
    dt = 0.3 * mesh.hmin()
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.plane_data(**data_kw), dt, precision=precision)
    wn, t, _ = s.solve(steps)
    err = s.error_l2()
    launches = s.launches
    s.close()
    rm = ref.RefMesh(c, e)
    r = rm.run(ref.SCHEME_RK3, ref.make_data(**data_kw), dt, steps)
    return wn, t, err, r, launches


@pytest.mark.parametrize("n,jitter,steps", [(2, 0.0, 10), (4, 0.15, 20), (8, 0.0, 200)])
def test_rk3_fp64_matches_reference(n, jitter, steps):
    kw = dict(khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0))
    wn, t, err, r, launches = _run_pair(n, jitter, steps, kw)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= FP64_RTOL, rel
    assert t == r["t"]
    assert abs(err - r["err"]) <= 1e-10 * r["err"]
    assert launches >= 3 * steps


def test_rk3_fp64_oblique_wave_matches_reference():
    k = np.array([1.0, 2.0, -0.5])
    k /= np.linalg.norm(k)
    p = np.cross(k, [0.0, 0.0, 1.0])
    p /= np.linalg.norm(p)
    kw = dict(khat=k, kmag=3 * np.pi, pol=p, amp=0.7, phase=0.3)
    wn, t, err, r, _ = _run_pair(4, 0.1, 30, kw, seed=11)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= FP64_RTOL, rel


def test_rk3_fp32_close_to_reference():
    kw = dict(khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0))
    wn, t, err, r, _ = _run_pair(8, 0.0, 200, kw, precision=capi.FP32)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    # FP32 storage and arithmetic over 600 stages: well under the
    # discretisation error (~5e-4 relative to the field at this size)
    assert rel <= 2e-5, rel
    assert abs(err - r["err"]) <= 0.01 * r["err"]


import os  # noqa: E402

from oracle import port  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["kuhn2", "kuhn3j"])
def test_rk3_fp64_matches_golden_fixture(name):
    """Against the committed vectors of the reference's own dg_solve_rk3
    (tests/golden/make_golden.py), with the reference's tables passed through
    the C-ABI as a reference host would."""
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {k[5:]: g[k] for k in g.files if k.startswith("mesh_")}
    mesh = capi.MeshArrays(arrays["face2elem"], arrays["fnode2enode"], arrays["boundaryface"],
                           arrays["elem2qnode"], arrays["node"], int(g["nbelems"]))
    tabs = capi.tables_from_numpy({k[4:]: g[k] for k in g.files if k.startswith("t10_")})
    p = g["plane"]
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.plane_data(khat=p[:3], kmag=p[3], pol=p[4:7]),
                    float(g["dt"]), tables=tabs)
    wn, t, _ = s.solve(int(g["rk3_steps"]))
    err = s.error_l2()
    s.close()
    rel = np.linalg.norm(wn - g["rk3_wn"]) / np.linalg.norm(g["rk3_wn"])
    assert rel <= FP64_RTOL, rel
    assert t == float(g["rk3_t"])
    assert abs(err - float(g["rk3_err"])) <= 1e-10 * float(g["rk3_err"])


def test_rk3_fp64_matches_oracle_16():
    c, e = kuhn.kuhn_cube(16, 0.15, seed=21)
    mesh = capi.mesh_build(c, e)
    dt = 0.3 * mesh.hmin()
    kw = dict(khat=(0.0, 0.6, 0.8), kmag=4 * np.pi, pol=(1.0, 0.0, 0.0))
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.plane_data(**kw), dt)
    wn, t, _ = s.solve(12)
    s.close()
    arrays = dict(face2elem=mesh.face2elem, fnode2enode=mesh.fnode2enode,
                  boundaryface=mesh.boundaryface, elem2qnode=mesh.elem2qnode, node=mesh.node)
    o = port.Oracle(mesh.nbelems, arrays, capi.tables_as_numpy(capi.t10_tables()))
    wo, to = o.rk3(port.Oracle.data(**kw), dt, 12)
    rel = np.linalg.norm(wn - wo) / np.linalg.norm(wo)
    assert rel <= FP64_RTOL, rel
    assert t == to


def test_rk3_step_host_equals_device_resident_steps():
    """gdn_cuda_step_host (host state in/out) gives the same state as
    advancing on the device."""
    c, e = kuhn.kuhn_cube(4, 0.1, seed=2)
    mesh = capi.mesh_build(c, e)
    dt = 0.3 * mesh.hmin()
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.plane_data(), dt)
    s.init()
    s.advance(3)
    w3 = s.get_state()
    t3 = s.t
    s.advance(4)
    w7 = s.get_state()
    host = w3.copy()
    s.set_state(host, t3)
    s.step_host(host, 4)
    s.close()
    assert np.array_equal(host[: 60 * mesh.nbelems], w7[: 60 * mesh.nbelems])


@pytest.mark.parametrize("scheme", [capi.SCHEME_RK3, capi.SCHEME_KINETIC])
def test_graph_replay_equals_direct_launches(scheme):
    """Step loops replayed from captured CUDA graphs launch the same kernels
    in the same order as direct launches: identical states and times."""
    c, e = kuhn.kuhn_cube(5, 0.1, seed=6)
    mesh = capi.mesh_build(c, e)
    dt = 0.3 * mesh.hmin() * (1 if scheme == capi.SCHEME_RK3 else 10)
    data = capi.plane_data() if scheme == capi.SCHEME_RK3 else capi.cavity_data()
    out = []
    for g in (0, 1):
        s = capi.Solver(mesh, scheme, data, dt, use_graph=g)
        wn, t, _ = s.solve(7)  # odd: graphs of 2 RK3 steps plus one direct step
        s.close()
        out.append((wn, t))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


@pytest.mark.parametrize("n,jitter", [(3, 0.0), (4, 0.15)])
def test_rk3_metal_boundary_matches_reference(n, jitter):
    """RK3 with the metal boundary flux (-n x H_L, 0) (maxwell.c:205-223) on
    the PEC cavity mode, against the reference built with
    maxwell_num_flux_boundary_metal as model->get_num_flux_boundary."""
    c, e = kuhn.kuhn_cube(n, jitter, seed=4)
    mesh = capi.mesh_build(c, e)
    dt = 0.3 * mesh.hmin()
    steps = 15
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.cavity_data(), dt, boundary_flux=capi.BC_METAL)
    wn, t, _ = s.solve(steps)
    err = s.error_l2()
    s.close()
    r = ref.RefMesh(c, e).run(ref.SCHEME_RK3_METAL, ref.make_data(kind=ref.DATA_CAVITY), dt, steps)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= FP64_RTOL, rel
    assert abs(err - r["err"]) <= 1e-10 * r["err"]
    # the metal flux differs from the upwind flux with the exact data
    s2 = capi.Solver(mesh, capi.SCHEME_RK3, capi.cavity_data(), dt)
    wu, _, _ = s2.solve(steps)
    s2.close()
    assert np.linalg.norm(wu - wn) > 1e-6 * np.linalg.norm(wn)


_REF15 = {}


def _ref15(kind):
    """The reference build on a 15^3 x 6 mesh (20250 tets: a partial last
    tile, and more tiles than a persistent grid holds), 20 steps."""
    if kind not in _REF15:
        c, e = kuhn.kuhn_cube(15, 0.1, seed=8)
        mesh = capi.mesh_build(c, e)
        dt = 0.3 * mesh.hmin()
        if kind == "plane":
            r = ref.RefMesh(c, e).run(ref.SCHEME_RK3, ref.make_data(khat=(0.6, 0.8, 0.0), kmag=4 * np.pi,
                                                                   pol=(0, 0, 1)), dt, 20)
        else:
            r = ref.RefMesh(c, e).run(ref.SCHEME_RK3_METAL, ref.make_data(kind=ref.DATA_CAVITY), dt, 20)
        _REF15[kind] = (mesh, dt, r)
    return _REF15[kind]


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("variant", [1, 2])
def test_rk3_every_stage_variant_matches_reference(variant, precision):
    """Each stage kernel variant (two register budgets and neighbour-trace
    prefetch modes) against the reference build."""
    mesh, dt, r = _ref15("plane")
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.plane_data(khat=(0.6, 0.8, 0.0), kmag=4 * np.pi, pol=(0, 0, 1)),
                    dt, precision=precision, rk3_variant=variant)
    assert s.rk3_variant[0] == variant
    wn, t, _ = s.solve(20)
    s.close()
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= (FP64_RTOL if precision == capi.FP64 else 2e-5), rel


@pytest.mark.parametrize("variant", [1, 2])
def test_rk3_variants_metal_boundary(variant):
    mesh, dt, r = _ref15("metal")
    s = capi.Solver(mesh, capi.SCHEME_RK3, capi.cavity_data(), dt, rk3_variant=variant, boundary_flux=capi.BC_METAL)
    wn, _, _ = s.solve(20)
    s.close()
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= FP64_RTOL, rel


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32])
def test_rk3_table_product_path_matches_reference(precision):
    """Tables without the tetrahedral symmetry the factored kernel relies on
    (one inverse-mass pair moved by 1e-13 of the largest entry, far below the
    FP64 tolerance but above the attach check's 1e-15) run the table-product
    kernel (structural zeros of D_k and of the face mass removed, derivatives
    exchanged through shared memory): still the reference's result."""
    mesh, dt, r = _ref15("plane")
    t = capi.t10_tables()
    d = 1e-13 * 600.0
    t.inv_mass[0][1] += d
    t.inv_mass[1][0] += d
    data = capi.plane_data(khat=(0.6, 0.8, 0.0), kmag=4 * np.pi, pol=(0, 0, 1))
    for v in (1, 2):
        s = capi.Solver(mesh, capi.SCHEME_RK3, data, dt, precision=precision, tables=t, rk3_variant=v)
        wn, _, _ = s.solve(20)
        s.close()
        rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
        assert rel <= (FP64_RTOL if precision == capi.FP64 else 2e-5), (v, rel)
