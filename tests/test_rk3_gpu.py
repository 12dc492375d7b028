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
