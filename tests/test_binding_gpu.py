"""The drop-in, end to end on the GPU: the reference's own flow on the
reference's own gmsh meshes, with dg_solve routed to the B200 path by the
compiled binding (integration/dg_cuda.c, linked into
oracle/_ref/libgdon3d_ref_bound.so by oracle/Makefile):

  mesh_read_from_msh22_file -> mesh_build_connectivity -> simulation_init
  -> simulation_set_time_parameters -> dg_cuda_attach -> dg_solve (GPU)
  -> simulation_error_l2

against the same flow through the unmodified reference (libgdon3d_ref_zero.so,
its dg_solve on the CPU).  Meshes: data/mesh/t4_cube_8.msh, t4_cube_16.msh,
t4_cube_8_torus_128.msh, written back from tests/golden/ref_meshes.npz.
Model setup as the reference's examples: the cos wave of
examples/rk3_maxwell_plane_wave.c:35-80 (RK3) and
examples/relax_maxwell_plane_wave.c:35-70 (d3q4), the stationary data of
examples/relax_maxwell_stationary_wave.c:31-45 (d3q4); the GPU descriptor of
the cos wave is the plane wave khat = (1,0,0), pol = (0,0,1), kmag = pi,
phase = pi/2, checked by the binding against the callback.

Bar: FP64 relative L2 of the whole state (boundary dofs included) <= 1e-12,
the same final time, the error norm within 1e-10 relative.
"""
import os

import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn
from oracle import ref

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_meshes.npz")
MESHES = ["t4_cube_8", "t4_cube_16", "t4_cube_8_torus_128"]
# the examples' time step (examples/rk3_maxwell_plane_wave.c:70-72)
EXAMPLE_DT = 0.032 * (1.0 / 9)


def example_cos_descriptor():
    return capi.plane_data(khat=(1.0, 0.0, 0.0), kmag=np.pi, pol=(0.0, 0.0, 1.0), phase=0.5 * np.pi)


@pytest.fixture(scope="module")
def msh_files(tmp_path_factory):
    g = np.load(GOLDEN)
    d = tmp_path_factory.mktemp("msh")
    out = {}
    for name in MESHES:
        p = str(d / (name + ".msh"))
        kuhn.write_msh22(p, g[name + "_coords"], g[name + "_elem2node"])
        out[name] = p
    return out


def _pair(path, scheme, data_kind, gpu_data, dt, steps, precision=capi.FP64):
    cpu = ref.RefMesh(path=path, variant="zero")
    r = cpu.run(scheme, ref.make_data(kind=data_kind), dt, steps)
    cpu.close()
    gm = ref.RefMesh(path=path, variant="bound")
    g = gm.run_bound(scheme, ref.make_data(kind=data_kind), gpu_data, dt, steps, precision)
    gm.close()
    assert g["rc"] == 0, g["msg"]
    return r, g


def _check(r, g):
    rel = np.linalg.norm(g["wn"] - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= FP64_RTOL, rel
    assert g["t"] == r["t"]
    assert abs(g["err"] - r["err"]) <= 1e-10 * r["err"], (g["err"], r["err"])
    assert g["mismatch"] <= 1e-14


@pytest.mark.parametrize("name", MESHES)
def test_rk3_reference_flow_on_reference_mesh(msh_files, name):
    path = msh_files[name]
    hmin = ref.RefMesh(path=path).hmin()
    r, g = _pair(path, ref.SCHEME_RK3, ref.DATA_EXAMPLE_COS, example_cos_descriptor(), 0.3 * hmin, 40)
    _check(r, g)


def test_rk3_reference_flow_at_the_examples_dt(msh_files):
    """t4_cube_8 at the examples' own dt (stable there; the finer meshes need
    the CFL step)."""
    r, g = _pair(msh_files["t4_cube_8"], ref.SCHEME_RK3, ref.DATA_EXAMPLE_COS, example_cos_descriptor(),
                 EXAMPLE_DT, 40)
    _check(r, g)


@pytest.mark.parametrize("name", MESHES)
def test_d3q4_reference_flow_on_reference_mesh(msh_files, name):
    r, g = _pair(msh_files[name], ref.SCHEME_D3Q4, ref.DATA_EXAMPLE_COS, example_cos_descriptor(), EXAMPLE_DT, 20)
    _check(r, g)


def test_d3q4_stationary_data_on_cube_16(msh_files):
    """examples/relax_maxwell_stationary_wave.c:31-45: maxwell_imposed_stationary,
    d3q4, t4_cube_16.msh, the examples' dt."""
    r, g = _pair(msh_files["t4_cube_16"], ref.SCHEME_D3Q4, ref.DATA_STATIONARY, capi.stationary_data(),
                 EXAMPLE_DT, 20)
    _check(r, g)


def test_d3q6_reference_flow_on_cube_8(msh_files):
    """The d3q6 velocity set (recognised by its get_feq, get_w and get_fR) through the
    binding, the examples' cos data."""
    r, g = _pair(msh_files["t4_cube_8"], ref.SCHEME_D3Q6, ref.DATA_EXAMPLE_COS, example_cos_descriptor(),
                 EXAMPLE_DT, 10)
    _check(r, g)


def test_rk3_metal_boundary_flux_on_cube_16(msh_files):
    """RK3 with maxwell_num_flux_boundary_metal as the model's boundary flux (the binding maps
    it to GDN_CUDA_BC_METAL), PEC cavity data, t4_cube_16."""
    path = msh_files["t4_cube_16"]
    hmin = ref.RefMesh(path=path).hmin()
    r, g = _pair(path, ref.SCHEME_RK3_METAL, ref.DATA_CAVITY, capi.cavity_data(), 0.3 * hmin, 30)
    _check(r, g)


@pytest.mark.parametrize("scheme,dt_rule,tmax_steps", [(ref.SCHEME_RK3, "cfl", 20), (ref.SCHEME_D3Q4, "example", 10)])
def test_reference_convergence_driver_routed_to_the_gpu(msh_files, scheme, dt_rule, tmax_steps):
    """dg_cuda_route_all, then the reference's own utils_l2_time_convergence
    (src/utils/convergence.c:43-104) on t4_cube_8.msh: the driver builds its own
    gdn_simulation and halves dt per run; every dg_solve it makes is attached on first use,
    attached again when dt changes, and solved on the GPU.  Its printed errors (12
    decimals) equal those of the unmodified reference's CPU run."""
    path = msh_files["t4_cube_8"]
    dt = 0.3 * ref.RefMesh(path=path).hmin() if dt_rule == "cfl" else EXAMPLE_DT
    d = ref.make_data(kind=ref.DATA_EXAMPLE_COS)
    cpu = ref.time_convergence(path, scheme, d, dt, tmax_steps * dt, 2, variant="zero")
    gpu = ref.time_convergence(path, scheme, d, dt, tmax_steps * dt, 2, variant="bound",
                               gpu_data=example_cos_descriptor())
    assert len(cpu) == 2 and len(gpu) == 2
    for a, b in zip(cpu, gpu):
        assert a["dt"] == b["dt"] and a["iter"] == b["iter"]
        assert abs(a["error"] - b["error"]) <= 2e-12 + 1e-10 * a["error"], (a, b)


def test_rk3_fp32_through_the_binding(msh_files):
    """The precision choice travels through the binding's config."""
    path = msh_files["t4_cube_16"]
    hmin = ref.RefMesh(path=path).hmin()
    r, g = _pair(path, ref.SCHEME_RK3, ref.DATA_EXAMPLE_COS, example_cos_descriptor(), 0.3 * hmin, 40,
                 precision=capi.FP32)
    rel = np.linalg.norm(g["wn"] - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 2e-5, rel
    assert abs(g["err"] - r["err"]) <= 0.01 * r["err"]


@pytest.mark.parametrize("scheme,kind,bad", [
    (ref.SCHEME_RK3, ref.DATA_EXAMPLE_COS, dict(kmag=2 * np.pi)),      # wrong frequency
    (ref.SCHEME_RK3, ref.DATA_EXAMPLE_COS, dict(phase=0.0)),           # sin instead of cos
    (ref.SCHEME_D3Q4, ref.DATA_STATIONARY, None),                      # plane wave for stationary data
])
def test_descriptor_that_differs_from_the_callback_is_refused(msh_files, scheme, kind, bad):
    kw = dict(khat=(1.0, 0.0, 0.0), kmag=np.pi, pol=(0.0, 0.0, 1.0), phase=0.5 * np.pi)
    if bad:
        kw.update(bad)
    gm = ref.RefMesh(path=msh_files["t4_cube_8"], variant="bound")
    g = gm.run_bound(scheme, ref.make_data(kind=kind), capi.plane_data(**kw), EXAMPLE_DT, 2)
    gm.close()
    assert g["rc"] == capi.ERR_INVALID
    assert "differs from get_imposed_data" in g["msg"]
    assert g["mismatch"] > 1e-3


def test_eval_data_matches_reference_callbacks():
    """gdn_cuda_eval_data (device code) against the reference's own
    maxwell_imposed_stationary / maxwell_imposed_macro_cavity on the host, at
    random points and times."""
    rng = np.random.default_rng(5)
    x = rng.uniform(-0.2, 1.2, (4000, 3))
    for kind, desc in ((ref.DATA_STATIONARY, capi.stationary_data()), (ref.DATA_CAVITY, capi.cavity_data()),
                       (ref.DATA_EXAMPLE_COS, example_cos_descriptor())):
        for t in (0.0, 0.37, 2.5):
            w_dev = capi.eval_data(desc, x, t)
            w_ref = ref.eval_callback(kind, x, t)
            scale = max(1.0, np.abs(w_ref).max())
            assert np.abs(w_dev - w_ref).max() <= 1e-14 * scale, (kind, t)
