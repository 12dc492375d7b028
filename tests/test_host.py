"""CPU: the C-ABI library loads and exports every symbol of
include/gdon3d_cuda.h; host-side logic (P2 tables, connectivity builder,
hmin, argument validation, mesh generator) against the reference's golden
fixtures.  No GPU compute is called here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gdon3d_b200 import capi, kuhn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "gdon3d_cuda.h")).read()
    declared = set(re.findall(r"\b(gdn_cuda_[a-z0-9_]+)\s*\(", hdr))
    assert declared, "no declarations found"
    L = capi.lib()
    for name in sorted(declared):
        assert hasattr(L, name), name
    assert declared == set(capi.EXPORTS)


def test_tables_match_reference_tables():
    g = _golden("kuhn2")
    t = capi.tables_as_numpy(capi.t10_tables())
    # face mass: the reference's 10-digit literals, bit for bit
    assert np.array_equal(t["face_scal"], g["t10_face_scal"])
    assert np.array_equal(t["face2node"], g["t10_face2node"])
    assert np.array_equal(t["mass"], g["t10_mass"])
    assert np.array_equal(t["inv_mass"], g["t10_inv_mass"])
    # exact rationals vs the reference's decimal literals: within 1 ulp (two
    # wpg entries, 1/sqrt(3) in the face-3 normal, 1e-18 noise in internal)
    for k in ("wpg", "internal", "ref_normal"):
        assert np.max(np.abs(t[k] - g["t10_" + k])) <= 2.3e-16, k


@pytest.mark.parametrize("name", ["kuhn2", "kuhn3j"])
def test_mesh_build_matches_reference_connectivity(name):
    g = _golden(name)
    m = capi.mesh_build(g["coords"], g["elem2node"])
    assert np.array_equal(m.face2elem, g["mesh_face2elem"])
    assert np.array_equal(m.fnode2enode, g["mesh_fnode2enode"])
    assert np.array_equal(m.boundaryface, g["mesh_boundaryface"])
    # P2 node ids are numbered differently; the coordinates of every
    # (element, local node) and boundary dof must be identical bit for bit
    x_ours = m.node.reshape(-1, 3)[m.elem2qnode]
    x_ref = g["mesh_node"].reshape(-1, 3)[g["mesh_elem2qnode"]]
    assert np.array_equal(x_ours, x_ref)
    assert m.hmin() == float(g["hmin"])


def test_mesh_build_rejects_bad_indices():
    c, e = kuhn.kuhn_cube(1)
    e = e.copy()
    e[0, 0] = 999
    with pytest.raises(capi.GdnError) as ex:
        capi.mesh_build(c, e)
    assert ex.value.code == capi.ERR_MESH


def test_attach_validates_before_touching_the_device():
    c, e = kuhn.kuhn_cube(2)
    m = capi.mesh_build(c, e)
    bad = capi.plane_data(khat=(1, 1, 0), pol=(0, 0, 1))  # not a unit vector
    with pytest.raises(capi.GdnError) as ex:
        capi.Solver(m, capi.SCHEME_RK3, bad, 0.01)
    assert ex.value.code == capi.ERR_INVALID
    with pytest.raises(capi.GdnError) as ex:
        capi.Solver(m, capi.SCHEME_RK3, capi.plane_data(), -1.0)
    assert ex.value.code == capi.ERR_INVALID
    with pytest.raises(capi.GdnError) as ex:
        capi.Solver(m, capi.SCHEME_KINETIC, capi.cavity_data(), 0.01, nb_v=5)
    assert ex.value.code == capi.ERR_UNSUPPORTED
    # corrupt connectivity: an element index out of range
    f2e = m.face2elem.copy()
    f2e[0] = 10 ** 6
    m2 = capi.MeshArrays(f2e, m.fnode2enode, m.boundaryface, m.elem2qnode, m.node, m.nbelems)
    with pytest.raises(capi.GdnError) as ex:
        capi.Solver(m2, capi.SCHEME_RK3, capi.plane_data(), 0.01)
    assert ex.value.code == capi.ERR_MESH
    assert "face2elem" in str(ex.value)


def test_null_handle_calls_fail_cleanly():
    L = capi.lib()
    assert L.gdn_cuda_advance(None, 1) == capi.ERR_INVALID
    assert L.gdn_cuda_detach(None) == capi.ERR_INVALID
    d = C.c_double()
    assert L.gdn_cuda_error_l2(None, C.byref(d)) == capi.ERR_INVALID
    assert b"bad arguments" in L.gdn_cuda_last_error()
    assert L.gdn_cuda_save_xdmf(None, 0, b"/nonexistent/x", 0) == capi.ERR_INVALID
    assert b"save_xdmf: bad arguments" in L.gdn_cuda_last_error()


@pytest.mark.parametrize("n,jitter", [(1, 0.0), (3, 0.0), (4, 0.15), (6, 0.3)])
def test_kuhn_mesh_is_conforming_and_positive(n, jitter):
    c, e = kuhn.kuhn_cube(n, jitter, seed=5)
    assert len(e) == 6 * n ** 3 and len(c) == (n + 1) ** 3
    p = c[e]
    det = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
    assert (det > 0).all()
    assert abs(det.sum() / 6.0 - 1.0) < 1e-12  # volumes tile the unit cube
    m = capi.mesh_build(c, e)
    assert m.nboundaryfaces == 12 * n * n
    assert m.nbfaces == (4 * len(e) + m.nboundaryfaces) // 2
    # boundary vertices never move
    on_b = (np.abs(c) < 1e-15) | (np.abs(c - 1) < 1e-15)
    assert on_b.any(axis=1).sum() == (n + 1) ** 3 - max(n - 1, 0) ** 3


def test_kuhn_jitter_is_seeded():
    a, _ = kuhn.kuhn_cube(4, 0.15, seed=9)
    b, _ = kuhn.kuhn_cube(4, 0.15, seed=9)
    c, _ = kuhn.kuhn_cube(4, 0.15, seed=10)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    base, _ = kuhn.kuhn_cube(4, 0.0)
    assert np.max(np.abs(a - base)) <= 0.15 / 4 + 1e-15


def test_msh22_roundtrip(tmp_path):
    c, e = kuhn.kuhn_cube(2, 0.1, seed=2)
    p = str(tmp_path / "m.msh")
    kuhn.write_msh22(p, c, e)
    c2, e2 = kuhn.read_msh22(p)
    assert np.array_equal(c, c2) and np.array_equal(e, e2)


def test_random_plane_wave_is_orthonormal():
    k, kmag, p = kuhn.random_plane_wave(3, 4 * np.pi)
    assert abs(np.linalg.norm(k) - 1) < 1e-15 and abs(np.linalg.norm(p) - 1) < 1e-15
    assert abs(np.dot(k, p)) < 1e-15 and kmag == 4 * np.pi


def test_batch_attach_validates_instances():
    """A batch needs one scheme (and one kinetic model) for all instances;
    the check happens before any device call."""
    c, e = kuhn.kuhn_cube(2)
    m = capi.mesh_build(c, e)
    L = capi.lib()
    tabs = capi.t10_tables()
    vi = np.zeros(3)
    rk3 = capi.Model(capi.SCHEME_RK3, 6, 0, 1.0, 0.0, capi._dp(vi), 0.5)
    vk = np.ascontiguousarray((capi.D3Q4_VI * capi.D3Q4_LAMBDA).ravel())
    kin = capi.Model(capi.SCHEME_KINETIC, 6, 4, capi.D3Q4_LAMBDA, capi.RELAX_OMEGA, capi._dp(vk), 0.5)
    d = capi.plane_data()
    inst = (capi.Instance * 2)()
    for i, mod in enumerate((rk3, kin)):
        inst[i].mesh = C.pointer(m.struct)
        inst[i].model = C.pointer(mod)
        inst[i].data = C.pointer(d)
        inst[i].dt = 0.01
    h = C.c_void_p()
    rc = L.gdn_cuda_attach_batch(inst, 2, C.byref(tabs), None, C.byref(h))
    assert rc == capi.ERR_UNSUPPORTED
    assert "one scheme" in L.gdn_cuda_last_error().decode()
    rc = L.gdn_cuda_attach_batch(inst, 0, C.byref(tabs), None, C.byref(h))
    assert rc == capi.ERR_INVALID


def test_convergence_drivers_validate_before_touching_the_device():
    c, e = kuhn.kuhn_cube(2)
    m = capi.mesh_build(c, e)
    with pytest.raises(capi.GdnError) as ex:
        capi.time_convergence(m, capi.SCHEME_RK3, capi.plane_data(), 0.1, 0.15, 2)  # tmax < 2 steps
    assert ex.value.code == capi.ERR_INVALID
    with pytest.raises(capi.GdnError) as ex:
        capi.time_convergence(m, capi.SCHEME_RK3, capi.plane_data(), 0.1, 1.0, 0)
    assert ex.value.code == capi.ERR_INVALID


def _p2_sums(x):
    edges = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]
    sv, se = x[:4].sum(), x[4:].sum()
    ev = np.array([sum(x[4 + e] for e, (a, b) in enumerate(edges) if l in (a, b)) for l in range(4)])
    return sv, se, ev, edges


@pytest.mark.parametrize("which", ["ours", "reference"])
def test_symmetric_table_forms_reproduce_the_table_products(which):
    """The factored RK3 kernel replaces three table products by sums over the
    P2 tetrahedron's symmetry (q4_apply_sym, lift_minv_sym, the face-mass lift)
    and the volume derivative by the P1-basis form (p1_weak_derivative).  The
    same algebra in numpy, against the dense products of the tables handed to
    attach (ours and the reference's)."""
    from oracle import ref
    if which == "ours":
        t = capi.tables_as_numpy(capi.t10_tables())
        D = t["internal"].reshape(10, 10, 3)
        M, Mi, S = t["mass"].reshape(10, 10), t["inv_mass"].reshape(10, 10), t["face_scal"].reshape(6, 6)
    else:
        t = ref.t10_tables()
        D, M, Mi, S = t["internal"], t["mass"], t["inv_mass"], t["face_scal"]
    rng = np.random.default_rng(7)
    x = rng.standard_normal(10)
    sv, se, ev, edges = _p2_sums(x)
    # Q4 = 4 Lambda M (lambda_l interpolated exactly in P2), vertex diagonal zero
    Lam = np.zeros((4, 10))
    for l in range(4):
        Lam[l, l] = 1.0
    for e, (a, b) in enumerate(edges):
        Lam[a, 4 + e] = Lam[b, 4 + e] = 0.5
    Q4 = 4.0 * Lam @ M
    for l in range(4):
        Q4[l, l] = 0.0
    qa, qb, qc = Q4[0, 1], Q4[0, 4], Q4[0, 5]
    v = (qa * sv + qc * se) - qa * x[:4] + (qb - qc) * ev
    assert np.abs(v - Q4 @ x).max() <= 1e-15 * np.abs(Q4 @ x).max() * 10
    assert abs((0.75 * qa * sv + 0.5 * (qb + qc) * se) - v.sum() / 4) <= 1e-15
    # weak derivative along g through the P1 basis == sum_k g_k D_k w
    g3 = rng.standard_normal(3)
    g = np.array([-g3.sum(), *g3])
    t4 = v - v.sum() / 4
    out = np.concatenate([g * t4, [g[a] * v[b] + g[b] * v[a] for a, b in edges]])
    dense = sum(g3[k] * (D[:, :, k] @ x) for k in range(3))
    assert np.abs(out - dense).max() <= 1e-14 * np.abs(dense).max()
    # Minv R through the symmetry
    m = [Mi[0, 1], Mi[0, 5], Mi[4, 9], Mi[0, 0] - Mi[0, 1], Mi[0, 4] - Mi[0, 5],
         Mi[4, 4] - 2 * Mi[4, 5] + Mi[4, 9], Mi[4, 5] - Mi[4, 9]]
    bv, be = m[0] * sv + m[1] * se, m[1] * sv + m[2] * se
    dw = np.concatenate([bv + m[3] * x[:4] + m[4] * ev,
                         [be + m[4] * (x[a] + x[b]) + m[5] * x[4 + e] + m[6] * (ev[a] + ev[b])
                          for e, (a, b) in enumerate(edges)]])
    assert np.abs(dw - Mi @ x).max() <= 1e-13 * np.abs(Mi @ x).max()
    # face mass on the triangle (vertices 0-2, edges 01, 12, 20)
    F = rng.standard_normal(6)
    s = [S[0, 0] - S[0, 1], S[0, 1], S[0, 4], S[3, 3] - S[3, 4], S[3, 4]]
    fo = np.zeros(6)
    for i in range(3):
        fo[i] = s[1] * F[:3].sum() + s[0] * F[i] + s[2] * F[3 + (i + 1) % 3]
    for k in range(3):
        fo[3 + k] = s[4] * F[3:].sum() + s[3] * F[3 + k] + s[2] * F[(k + 2) % 3]
    assert np.abs(fo - S @ F).max() <= 1e-15 * np.abs(S @ F).max() * 10


def _rk3_tix(e, k):
    return ((e >> 5) * 60 + k) * 32 + (e & 31)


@pytest.mark.parametrize("ne", [1, 31, 32, 33, 1000, 5308416, 71_582_784])
def test_rk3_gather_and_prefetch_offsets_stay_in_bounds(ne):
    """Index arithmetic of the RK3 stage kernel, restated: the 32-bit
    neighbour-trace offset used when the tiled state fits 32 bits equals the
    64-bit tiled index, every trace read (6 fields, stride 32) lies inside the
    ntiles * 1920 values allocated, and the L2 prefetch of a tile covers only
    allocated rows (state / k2 / geometry padded to whole tiles, neighbour and
    permutation rows only for live elements)."""
    nt = (ne + 31) // 32
    idx32 = nt * 1920 <= 0xFFFFFFFF
    rng = np.random.default_rng(ne)
    nbv = np.unique(np.concatenate([[0, ne - 1], rng.integers(0, ne, 200)]))
    for qn in range(10):
        k64 = np.array([_rk3_tix(int(v), qn * 6) for v in nbv])
        assert (k64 + 5 * 32 < nt * 1920).all()
        if idx32:
            k32 = ((nbv.astype(np.uint64) >> 5) * 1920 + qn * 192 + (nbv.astype(np.uint64) & 31)) & 0xFFFFFFFF
            assert np.array_equal(k32.astype(np.int64), k64)
    assert idx32 == (ne <= 71_582_784)
    for tn in (0, nt - 1):
        live = min(32, ne - tn * 32)
        assert 1 <= live <= 32
        assert tn * 1920 + 1920 <= nt * 1920 and tn * 320 + 320 <= nt * 320
        assert tn * 32 * 4 + live * 4 <= 4 * ne  # nb / perm ints (16 bytes per element)
