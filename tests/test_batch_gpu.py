"""Batched solves (gdn_cuda_attach_batch): instances of uneven size, with
their own wave data and time steps, concatenated in one handle.  Every
element / sweep item does the same arithmetic as in a single-instance run, so
each instance's state must equal its own single-instance solve bit for bit."""
import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn

pytestmark = pytest.mark.gpu


def _instances(scheme):
    specs = [(3, 0.1, 1), (4, 0.0, 2), (2, 0.15, 3)]
    meshes, datas, dts = [], [], []
    for k, (n, jitter, seed) in enumerate(specs):
        c, e = kuhn.kuhn_cube(n, jitter, seed=seed)
        m = capi.mesh_build(c, e)
        meshes.append(m)
        if scheme == capi.SCHEME_KINETIC and k == 1:
            datas.append(capi.cavity_data())
        else:
            rng = np.random.default_rng(seed)
            kh = rng.standard_normal(3)
            kh /= np.linalg.norm(kh)
            pol = np.cross(kh, [0.3, 0.5, 0.7])
            pol /= np.linalg.norm(pol)
            datas.append(capi.plane_data(khat=kh, kmag=2 * np.pi * (1 + k), pol=pol))
        mult = 1 if scheme == capi.SCHEME_RK3 else 10
        dts.append(mult * 0.3 * m.hmin())
    return meshes, datas, dts


@pytest.mark.parametrize("scheme,precision", [(capi.SCHEME_RK3, capi.FP64), (capi.SCHEME_RK3, capi.FP32),
                                              (capi.SCHEME_KINETIC, capi.FP64),
                                              (capi.SCHEME_KINETIC, capi.FP32)])
def test_batch_equals_single_instance_solves(scheme, precision):
    meshes, datas, dts = _instances(scheme)
    steps = 5
    # one RK3 stage-kernel variant for both runs: the autotuner may pick
    # different ones for the batch and the single meshes
    b = capi.BatchSolver(meshes, datas, dts, scheme=scheme, precision=precision, rk3_variant=1)
    assert b.ninst == 3
    wn, t0, _ = b.solve(steps)
    errs = b.error_l2_batch()
    parts = b.split(wn)
    times = [b.instance_info(i)[0] for i in range(3)]
    b.close()
    for i in range(3):
        s = capi.Solver(meshes[i], scheme, datas[i], dts[i], precision=precision, rk3_variant=1)
        wi, ti, _ = s.solve(steps)
        ei = s.error_l2()
        s.close()
        assert np.array_equal(parts[i], wi), i
        assert times[i] == ti
        assert errs[i] == ei
    assert t0 == times[0]


def test_batch_set_get_state_round_trip():
    meshes, datas, dts = _instances(capi.SCHEME_KINETIC)
    b = capi.BatchSolver(meshes, datas, dts, scheme=capi.SCHEME_KINETIC)
    rng = np.random.default_rng(0)
    wn = rng.standard_normal(b.wlen)
    b.set_state(wn, 0.0)
    back = b.get_state()
    masks = []
    for i in range(b.ninst):
        _, ne, off, ln = b.instance_info(i)
        m = np.zeros(ln, bool).reshape(6 * b.nb_v, -1)
        m[:, : 10 * ne] = True
        masks.append(m.ravel())
    b.close()
    m = np.concatenate(masks)
    assert np.array_equal(back[m], wn[m])
