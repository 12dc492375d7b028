"""Convergence-study drivers (utils_l2_time_convergence /
utils_l2_space_convergence, src/utils/convergence.c) on the device: each run's
error equals the reference build's dg_solve + simulation_error_l2 at the same
dt and step count, and the orders follow from the errors."""
import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,refs,mult", [(capi.SCHEME_RK3, ref.SCHEME_RK3, 1.0),
                                              (capi.SCHEME_KINETIC, ref.SCHEME_D3Q4, 10.0)])
def test_time_convergence_matches_reference_runs(scheme, refs, mult):
    c, e = kuhn.kuhn_cube(3, 0.1, seed=2)
    mesh = capi.mesh_build(c, e)
    init_dt = mult * 0.3 * mesh.hmin()
    tmax = 9.5 * init_dt
    kw = dict(khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0))
    out = capi.time_convergence(mesh, scheme, capi.plane_data(**kw), init_dt, tmax, 3)
    assert list(out["iter"]) == [8, 16, 32]
    assert np.allclose(out["dt"], init_dt / np.array([1, 2, 4]), rtol=0, atol=0)
    rm = ref.RefMesh(c, e)
    for k in range(3):
        r = rm.run(refs, ref.make_data(**kw), out["dt"][k], int(out["iter"][k]))
        assert abs(out["err"][k] - r["err"]) <= 1e-10 * r["err"], (k, out["err"][k], r["err"])
    assert out["order"][0] == -1.0
    for k in (1, 2):
        assert out["order"][k] == pytest.approx(np.log(out["err"][k - 1] / out["err"][k]) / np.log(2.0))


def test_space_convergence_rk3_matches_reference_runs():
    meshes, cs = [], []
    for n in (2, 4):
        c, e = kuhn.kuhn_cube(n, 0.0, seed=1)
        cs.append((c, e))
        meshes.append(capi.mesh_build(c, e))
    init_dt = 0.3 * meshes[0].hmin()
    tmax = 6.5 * init_dt
    kw = dict(khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0))
    out = capi.space_convergence(meshes, capi.SCHEME_RK3, capi.plane_data(**kw), init_dt, tmax)
    assert list(out["iter"]) == [5, 10]
    assert out["hmin"][0] == pytest.approx(2 * out["hmin"][1])
    for k, (c, e) in enumerate(cs):
        r = ref.RefMesh(c, e).run(ref.SCHEME_RK3, ref.make_data(**kw), out["dt"][k], int(out["iter"][k]))
        assert abs(out["err"][k] - r["err"]) <= 1e-10 * r["err"]
    assert out["err"][1] < out["err"][0]
    assert out["order"][1] == pytest.approx(np.log(out["err"][0] / out["err"][1]) / np.log(out["hmin"][0] / out["hmin"][1]))
