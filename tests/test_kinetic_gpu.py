"""HP-2 parity on the GPU: the CFL-less kinetic step (level-scheduled block
sweeps + relaxation) against the reference's dg_solve_relaxation compiled from
its own sources (the sparse LU is the repo's exact direct-solve shim; parity
against KLU itself is unpinned because KLU is not installed)."""
import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn
from oracle import ref

pytestmark = pytest.mark.gpu


def _pair(n, jitter, steps, cfl_mult, nb_v=4, data="cavity", precision=capi.FP64, seed=5):
    c, e = kuhn.kuhn_cube(n, jitter, seed=seed)
    mesh = capi.mesh_build(c, e)
    dt = cfl_mult * 0.3 * mesh.hmin()
    if data == "cavity":
        gd, rd = capi.cavity_data(), ref.make_data(kind=ref.DATA_CAVITY)
    else:
        kw = dict(khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0))
        gd, rd = capi.plane_data(**kw), ref.make_data(**kw)
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, gd, dt, nb_v=nb_v, precision=precision)
    wn, t, _ = s.solve(steps)
    err = s.error_l2()
    levels = s.num_levels
    s.close()
    r = ref.RefMesh(c, e).run(ref.SCHEME_D3Q4 if nb_v == 4 else ref.SCHEME_D3Q6, rd, dt, steps)
    return wn, t, err, r, levels


@pytest.mark.parametrize("n,jitter,steps,mult", [(2, 0.0, 5, 10), (4, 0.15, 10, 10), (4, 0.0, 10, 20)])
def test_kinetic_d3q4_fp64_matches_reference(n, jitter, steps, mult):
    wn, t, err, r, levels = _pair(n, jitter, steps, mult)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 1e-12, rel
    assert t == r["t"]
    assert abs(err - r["err"]) <= 1e-10 * r["err"]
    assert levels >= 1


def test_kinetic_d3q6_plane_fp64_matches_reference():
    wn, t, err, r, _ = _pair(3, 0.1, 6, 10, nb_v=6, data="plane")
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 1e-12, rel


def test_kinetic_cavity_16_fp64_matches_reference():
    """The plain CFL-less relaxation workload: 16^3 x 6 tets, PEC cavity mode,
    dt = 10 x the RK3 CFL step, 100 steps, d3q4."""
    wn, t, err, r, levels = _pair(16, 0.0, 100, 10)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 1e-12, rel
    assert abs(err - r["err"]) <= 1e-10 * r["err"]


def test_kinetic_fp32_close_to_reference():
    wn, t, err, r, _ = _pair(8, 0.0, 20, 10, precision=capi.FP32)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 1e-4, rel
    assert abs(err - r["err"]) <= 0.01 * r["err"]


import os  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name,nb_v", [("kuhn2", 4), ("kuhn3j", 4), ("kuhn2", 6)])
def test_kinetic_fp64_matches_golden_fixture(name, nb_v):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {k[5:]: g[k] for k in g.files if k.startswith("mesh_")}
    mesh = capi.MeshArrays(arrays["face2elem"], arrays["fnode2enode"], arrays["boundaryface"],
                           arrays["elem2qnode"], arrays["node"], int(g["nbelems"]))
    tabs = capi.tables_from_numpy({k[4:]: g[k] for k in g.files if k.startswith("t10_")})
    if nb_v == 4:
        data, key = capi.cavity_data(), "q4"
    else:
        p = g["plane"]
        data, key = capi.plane_data(khat=p[:3], kmag=p[3], pol=p[4:7]), "q6"
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, data, 10 * float(g["dt"]), nb_v=nb_v, tables=tabs)
    wn, t, _ = s.solve(int(g[key + "_steps"]))
    s.close()
    rel = np.linalg.norm(wn - g[key + "_wn"]) / np.linalg.norm(g[key + "_wn"])
    assert rel <= 1e-12, rel
    assert t == float(g[key + "_t"])


def _vol_mask(s, mesh):
    """True on the volume dofs of the kinetic reference layout
    wn[(iw * nb_v + iv) * neq + ipg] (ipg < 10 * nbelems)."""
    neq = s.wlen // (6 * s.nb_v)
    m = np.zeros((6 * s.nb_v, neq), bool)
    m[:, : 10 * mesh.nbelems] = True
    return m.ravel()


def test_kinetic_state_round_trip_through_sweep_order():
    """set_state scatters the reference layout into the device's sweep order
    and get_state gathers it back: volume dofs come back bit for bit."""
    c, e = kuhn.kuhn_cube(5, 0.1, seed=4)
    mesh = capi.mesh_build(c, e)
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), 3 * mesh.hmin(), nb_v=6)
    rng = np.random.default_rng(3)
    wn = rng.standard_normal(s.wlen)
    s.set_state(wn, 0.25)
    back = s.get_state()
    m = _vol_mask(s, mesh)
    s.close()
    assert np.array_equal(back[m], wn[m])


def test_kinetic_step_host_equals_device_resident_steps():
    """gdn_cuda_step_host (host state in/out) gives the same state as
    advancing on the device."""
    c, e = kuhn.kuhn_cube(4, 0.1, seed=2)
    mesh = capi.mesh_build(c, e)
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), 3 * mesh.hmin())
    s.init()
    s.advance(3)
    w3 = s.get_state()
    t3 = s.t
    s.advance(4)
    w7 = s.get_state()
    host = w3.copy()
    s.set_state(host, t3)
    s.step_host(host, 4)
    m = _vol_mask(s, mesh)
    s.close()
    assert np.array_equal(host[m], w7[m])


def _variants(nb_v, n=6, jitter=0.15, mult=10, steps=10):
    c, e = kuhn.kuhn_cube(n, jitter, seed=3)
    mesh = capi.mesh_build(c, e)
    dt = mult * 0.3 * mesh.hmin()
    out = {}
    for name, prec, passes in [("fp64", capi.FP64, 1), ("fp32", capi.FP32, 1), ("ref1", capi.FP32_REFINE, 1),
                               ("ref2", capi.FP32_REFINE, 2), ("bf16", capi.BF16_STORE, 1)]:
        s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), dt, nb_v=nb_v, precision=prec,
                        refine_passes=passes)
        wn, t, _ = s.solve(steps)
        out[name] = (wn, s.error_l2())
        s.close()
    return out


@pytest.mark.parametrize("nb_v", [4, 6])
def test_kinetic_fp32_refinement_recovers_fp64(nb_v):
    """FP32 sweeps plus FP64-residual refinement: each pass multiplies the
    distance to the FP64 solve by ~1e-6 (FP32 sweeps alone: ~1e-6)."""
    out = _variants(nb_v)
    ref = out["fp64"][0]
    rel = {k: np.linalg.norm(v[0] - ref) / np.linalg.norm(ref) for k, v in out.items()}
    assert 1e-8 < rel["fp32"] < 1e-5, rel
    assert rel["ref1"] <= 1e-11, rel
    assert rel["ref2"] <= 1e-13, rel
    assert rel["ref2"] < rel["ref1"] < rel["fp32"]
    # the analytic error of the refined runs is the FP64 one
    assert abs(out["ref1"][1] - out["fp64"][1]) <= 1e-9 * out["fp64"][1]


def test_kinetic_bf16_storage_error_is_bounded():
    """BF16 distributions with FP32 arithmetic: the state stays within a few
    1e-3 of the FP64 run on a coarse mesh (BF16 keeps 8 significant bits)."""
    out = _variants(4)
    ref = out["fp64"][0]
    rel = np.linalg.norm(out["bf16"][0] - ref) / np.linalg.norm(ref)
    assert 1e-4 < rel < 2e-2, rel
    assert abs(out["bf16"][1] - out["fp64"][1]) <= 0.1 * out["fp64"][1]


@pytest.mark.parametrize("precision,nb_v", [(capi.FP64, 4), (capi.FP32, 6), (capi.FP32_REFINE, 4),
                                            (capi.BF16_STORE, 4)])
def test_kinetic_sweep_modes_equal_level_launches(precision, nb_v):
    """One cooperative launch walking all sweep levels (grid barrier between
    levels), one flag-driven launch (each chunk waits for its upwind
    neighbours' readiness flags) and one cooperative launch of spatial parts
    (each CTA sweeps its part, waiting only for other parts' items) do per
    item the arithmetic of one launch per level: identical states."""
    c, e = kuhn.kuhn_cube(5, 0.15, seed=8)
    mesh = capi.mesh_build(c, e)
    dt = 10 * 0.3 * mesh.hmin()
    out = []
    for mode in (1, 2, 3, 4):
        s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), dt, precision=precision, nb_v=nb_v,
                        kin_sweep=mode)
        assert s.kin_sweep_mode == mode
        wn, t, _ = s.solve(6)
        out.append((wn, t, s.error_l2()))
        s.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0])
        assert out[0][1] == o[1] and out[0][2] == o[2]


@pytest.mark.parametrize("mode", [3, 4])
def test_kinetic_one_launch_sweeps_cavity_16_match_reference(mode):
    """The flag-driven and the spatial-parts sweeps on the plain CFL-less
    workload (16^3 x 6 cavity, 10 x CFL, d3q4) against the reference build,
    30 steps."""
    c, e = kuhn.kuhn_cube(16, 0.0, seed=5)
    mesh = capi.mesh_build(c, e)
    dt = 10 * 0.3 * mesh.hmin()
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), dt, kin_sweep=mode)
    assert s.kin_sweep_mode == mode
    wn, t, _ = s.solve(30)
    s.close()
    r = ref.RefMesh(c, e).run(ref.SCHEME_D3Q4, ref.make_data(kind=ref.DATA_CAVITY), dt, 30)
    rel = np.linalg.norm(wn - r["wn"]) / np.linalg.norm(r["wn"])
    assert rel <= 1e-12, rel
    assert t == r["t"]


@pytest.mark.parametrize("mode", [2, 3, 4])
def test_kinetic_bounded_wait_gives_up_with_timeout_status(mode):
    """A device-side wait whose limit runs out ends its launch and reports
    GDN_CUDA_ERR_TIMEOUT at the next call that reads the state; the context
    stays usable and, with the limit restored, the same handle solves
    correctly.  The limit is 0 polls: every wait whose condition is not met
    at its first poll gives up, which on a mesh of 80 sweep levels happens in
    the first levels (a flag that is not yet set, or CTAs still to arrive; the
    spatial-parts sweep has several hundred parts, most of them downstream of
    others)."""
    c, e = kuhn.kuhn_cube(12, 0.1, seed=3)
    mesh = capi.mesh_build(c, e)
    dt = 10 * 0.3 * mesh.hmin()
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), dt, kin_sweep=mode)
    assert s.num_levels > 40
    s.set_wait_limit(0)
    s.init()
    s.advance(3)
    with pytest.raises(capi.GdnError) as ex:
        s.get_state()
    assert ex.value.code == capi.ERR_TIMEOUT
    s.set_wait_limit(1 << 21)
    wn, t, _ = s.solve(3)
    s.close()
    s1 = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), dt, kin_sweep=1)
    w1, t1, _ = s1.solve(3)
    s1.close()
    assert np.array_equal(wn, w1) and t == t1


@pytest.mark.parametrize("n,levels", [(16, 108), (64, 444)])
def test_kinetic_device_schedule_levels(n, levels):
    """The device-built level schedule has the depth of the upwind DAG that
    Kahn's algorithm gives on the host for these Kuhn meshes (d3q4)."""
    c, e = kuhn.kuhn_cube(n, 0.0, seed=1)
    mesh = capi.mesh_build(c, e)
    s = capi.Solver(mesh, capi.SCHEME_KINETIC, capi.cavity_data(), 3 * mesh.hmin(), precision=capi.FP32,
                    kin_sweep=1)
    assert s.num_levels == levels
    s.close()
