"""ctypes bindings of include/gdon3d_cuda.h (libgdon3d_cuda.so, built in-tree).

This is the call a C99 host makes, restated for Python callers (tests and the
benchmark).  The library is loaded from this directory only; if it is missing
the import fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgdon3d_cuda.so")

OK = 0
ERR_CUDA, ERR_INVALID, ERR_UNSUPPORTED, ERR_CYCLE, ERR_OOM, ERR_TIMEOUT, ERR_MESH = 1, 2, 3, 4, 5, 6, 7
DATA_PLANE, DATA_CAVITY, DATA_STATIONARY = 0, 1, 2
SCHEME_RK3, SCHEME_KINETIC = 0, 1
BC_UPWIND, BC_METAL = 0, 1
FP64, FP32, FP32_REFINE, BF16_STORE = 0, 1, 2, 3

# d3q4 / d3q6 velocity sets (src/models/d3q4.c:17-24, src/models/d3q6.c:18-24)
D3Q4_LAMBDA = 1.732050807568877293
D3Q4_VI = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float64)
D3Q6_LAMBDA = 3.0
D3Q6_VI = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]],
                   dtype=np.float64)
RELAX_OMEGA = 1.999999999999


class GdnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("gdon3d_cuda error %d: %s" % (code, msg))
        self.code = code


class Mesh(C.Structure):
    _fields_ = [("nbelems", C.c_int), ("nbfaces", C.c_int), ("nboundaryfaces", C.c_int),
                ("nbqnodes", C.c_int), ("face2elem", C.POINTER(C.c_int)),
                ("fnode2enode", C.POINTER(C.c_int)), ("boundaryface", C.POINTER(C.c_int)),
                ("elem2qnode", C.POINTER(C.c_int)), ("node", C.POINTER(C.c_double))]


class Tables(C.Structure):
    _fields_ = [("wpg", C.c_double * 10), ("mass", (C.c_double * 10) * 10),
                ("inv_mass", (C.c_double * 10) * 10), ("internal", ((C.c_double * 3) * 10) * 10),
                ("face_scal", (C.c_double * 6) * 6), ("ref_normal", (C.c_double * 3) * 4),
                ("face2node", (C.c_int * 6) * 4)]


class Data(C.Structure):
    _fields_ = [("kind", C.c_int), ("khat", C.c_double * 3), ("kmag", C.c_double),
                ("pol", C.c_double * 3), ("amp", C.c_double), ("phase", C.c_double)]


class Model(C.Structure):
    _fields_ = [("scheme", C.c_int), ("nb_w", C.c_int), ("nb_v", C.c_int), ("lambda_", C.c_double),
                ("omega", C.c_double), ("vi", C.POINTER(C.c_double)), ("theta", C.c_double),
                ("boundary_flux", C.c_int)]


class Instance(C.Structure):
    _fields_ = [("mesh", C.POINTER(Mesh)), ("model", C.POINTER(Model)), ("data", C.POINTER(Data)),
                ("dt", C.c_double)]


class Config(C.Structure):
    _fields_ = [("precision", C.c_int), ("refine_passes", C.c_int), ("rk3_variant", C.c_int),
                ("use_graph", C.c_int), ("device", C.c_int), ("kin_sweep", C.c_int)]


EXPORTS = [
    "gdn_cuda_t10_tables", "gdn_cuda_mesh_build", "gdn_cuda_mesh_hmin", "gdn_cuda_attach",
    "gdn_cuda_detach", "gdn_cuda_solve", "gdn_cuda_init", "gdn_cuda_advance",
    "gdn_cuda_set_state", "gdn_cuda_get_state", "gdn_cuda_step_host", "gdn_cuda_error_l2",
    "gdn_cuda_get_time", "gdn_cuda_state_size", "gdn_cuda_num_levels", "gdn_cuda_launch_count",
    "gdn_cuda_stream", "gdn_cuda_last_error", "gdn_cuda_error_l2_noalloc", "gdn_cuda_attach_batch",
    "gdn_cuda_error_l2_batch", "gdn_cuda_num_instances", "gdn_cuda_instance_info", "gdn_cuda_rk3_variant",
    "gdn_cuda_kin_sweep_mode", "gdn_cuda_time_convergence", "gdn_cuda_space_convergence",
    "gdn_cuda_mesh_build_gpu", "gdn_cuda_save_xdmf", "gdn_cuda_eval_data",
    "gdn_cuda_set_wait_limit",
]

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libgdon3d_cuda.so is not built (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    ip, dp, vp = C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p
    L.gdn_cuda_last_error.restype = C.c_char_p
    L.gdn_cuda_t10_tables.argtypes = [C.POINTER(Tables)]
    L.gdn_cuda_mesh_build.argtypes = [C.c_int, dp, C.c_int, ip, ip, ip, ip, ip, ip, ip, ip, dp]
    L.gdn_cuda_mesh_hmin.argtypes = [C.POINTER(Mesh), dp]
    L.gdn_cuda_save_xdmf.argtypes = [vp, C.c_int, C.c_char_p, C.c_int]
    L.gdn_cuda_mesh_build_gpu.argtypes = [C.c_int, dp, C.c_int, ip, ip, ip, ip, ip, ip, ip, ip, dp, C.c_int]
    L.gdn_cuda_attach.argtypes = [C.POINTER(Mesh), C.POINTER(Tables), C.POINTER(Model),
                                  C.POINTER(Data), C.POINTER(Config), C.c_double, C.POINTER(vp)]
    L.gdn_cuda_detach.argtypes = [vp]
    L.gdn_cuda_solve.argtypes = [vp, C.c_int, dp, dp, dp]
    L.gdn_cuda_init.argtypes = [vp]
    L.gdn_cuda_advance.argtypes = [vp, C.c_int]
    L.gdn_cuda_set_state.argtypes = [vp, dp, C.c_double]
    L.gdn_cuda_get_state.argtypes = [vp, dp]
    L.gdn_cuda_step_host.argtypes = [vp, dp, C.c_int]
    L.gdn_cuda_error_l2.argtypes = [vp, dp]
    L.gdn_cuda_get_time.argtypes = [vp, dp]
    L.gdn_cuda_state_size.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gdn_cuda_num_levels.argtypes = [vp, ip]
    L.gdn_cuda_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.gdn_cuda_stream.argtypes = [vp, C.POINTER(vp)]
    L.gdn_cuda_error_l2_noalloc.argtypes = [vp, vp, vp, C.c_longlong, dp, C.POINTER(Data),
                                            C.c_double, vp, dp]
    L.gdn_cuda_attach_batch.argtypes = [C.POINTER(Instance), C.c_int, C.POINTER(Tables), C.POINTER(Config),
                                        C.POINTER(vp)]
    L.gdn_cuda_error_l2_batch.argtypes = [vp, dp]
    L.gdn_cuda_num_instances.argtypes = [vp, ip]
    L.gdn_cuda_rk3_variant.argtypes = [vp, ip, ip]
    L.gdn_cuda_kin_sweep_mode.argtypes = [vp, ip]
    L.gdn_cuda_time_convergence.argtypes = [C.POINTER(Mesh), C.POINTER(Tables), C.POINTER(Model), C.POINTER(Data),
                                            C.POINTER(Config), C.c_double, C.c_double, C.c_int, dp, ip, dp, dp]
    L.gdn_cuda_space_convergence.argtypes = [C.POINTER(C.POINTER(Mesh)), C.c_int, C.POINTER(Tables),
                                             C.POINTER(Model), C.POINTER(Data), C.POINTER(Config), C.c_double,
                                             C.c_double, C.c_int, dp, ip, dp, dp, dp]
    L.gdn_cuda_set_wait_limit.argtypes = [vp, C.c_longlong]
    L.gdn_cuda_eval_data.argtypes = [C.POINTER(Data), C.c_longlong, dp, C.c_double, dp, C.c_int]
    L.gdn_cuda_instance_info.argtypes = [vp, C.c_int, dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                         C.POINTER(C.c_longlong)]
    _lib = L
    return L


def check(rc: int):
    if rc != OK:
        raise GdnError(rc, lib().gdn_cuda_last_error().decode(errors="replace"))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def t10_tables() -> Tables:
    t = Tables()
    check(lib().gdn_cuda_t10_tables(C.byref(t)))
    return t


def tables_as_numpy(t: Tables) -> dict:
    return dict(wpg=np.ctypeslib.as_array(t.wpg).copy(),
                mass=np.ctypeslib.as_array(t.mass).copy(),
                inv_mass=np.ctypeslib.as_array(t.inv_mass).copy(),
                internal=np.ctypeslib.as_array(t.internal).copy(),
                face_scal=np.ctypeslib.as_array(t.face_scal).copy(),
                ref_normal=np.ctypeslib.as_array(t.ref_normal).copy(),
                face2node=np.ctypeslib.as_array(t.face2node).copy())


def tables_from_numpy(d: dict) -> Tables:
    t = Tables()
    np.ctypeslib.as_array(t.wpg)[:] = d["wpg"]
    np.ctypeslib.as_array(t.mass)[:] = d["mass"]
    np.ctypeslib.as_array(t.inv_mass)[:] = d["inv_mass"]
    np.ctypeslib.as_array(t.internal)[:] = d["internal"]
    np.ctypeslib.as_array(t.face_scal)[:] = d["face_scal"]
    np.ctypeslib.as_array(t.ref_normal)[:] = d["ref_normal"]
    np.ctypeslib.as_array(t.face2node)[:] = d["face2node"]
    return t


class MeshArrays:
    """The reference's connectivity arrays (the gdn_mesh fields the path
    consumes), kept alive for the Mesh struct that points into them."""

    def __init__(self, face2elem, fnode2enode, boundaryface, elem2qnode, node, nbelems):
        self.face2elem = np.ascontiguousarray(face2elem, dtype=np.int32)
        self.fnode2enode = np.ascontiguousarray(fnode2enode, dtype=np.int32)
        self.boundaryface = np.ascontiguousarray(boundaryface, dtype=np.int32)
        self.elem2qnode = np.ascontiguousarray(elem2qnode, dtype=np.int32)
        self.node = np.ascontiguousarray(node, dtype=np.float64)
        self.nbelems = int(nbelems)
        self.nbfaces = len(self.face2elem) // 4
        self.nboundaryfaces = len(self.boundaryface)
        self.nbqnodes = len(self.node) // 3
        bf = self.boundaryface if self.nboundaryfaces else np.zeros(1, np.int32)
        self._bf = bf
        self.struct = Mesh(self.nbelems, self.nbfaces, self.nboundaryfaces, self.nbqnodes,
                           _ip(self.face2elem), _ip(self.fnode2enode), _ip(bf),
                           _ip(self.elem2qnode), _dp(self.node))

    @property
    def neq(self) -> int:
        return 10 * self.nbelems + 6 * self.nboundaryfaces

    def hmin(self) -> float:
        h = C.c_double()
        check(lib().gdn_cuda_mesh_hmin(C.byref(self.struct), C.byref(h)))
        return h.value


def mesh_build(coords: np.ndarray, elem2node: np.ndarray, device=None) -> MeshArrays:
    """mesh_build_connectivity-equivalent arrays from T4 vertices (0-based),
    on the host (device=None) or on CUDA device `device` (same arrays)."""
    c = np.ascontiguousarray(coords, dtype=np.float64)
    e = np.ascontiguousarray(elem2node, dtype=np.int32)
    L = lib()
    if device is None:
        call = L.gdn_cuda_mesh_build
        extra = ()
    else:
        call = L.gdn_cuda_mesh_build_gpu
        extra = (int(device),)
    nf, nbf, nq = C.c_int(), C.c_int(), C.c_int()
    null_i = C.POINTER(C.c_int)()
    null_d = C.POINTER(C.c_double)()
    check(call(len(c), _dp(c), len(e), _ip(e), C.byref(nf), C.byref(nbf), C.byref(nq), null_i, null_i, null_i,
               null_i, null_d, *extra))
    f2e = np.zeros(4 * nf.value, np.int32)
    fn = np.zeros(12 * nf.value, np.int32)
    bf = np.zeros(max(nbf.value, 1), np.int32)
    e2q = np.zeros(10 * len(e) + 6 * nbf.value, np.int32)
    node = np.zeros(3 * nq.value, np.float64)
    check(call(len(c), _dp(c), len(e), _ip(e), C.byref(nf), C.byref(nbf), C.byref(nq), _ip(f2e), _ip(fn), _ip(bf),
               _ip(e2q), _dp(node), *extra))
    return MeshArrays(f2e, fn, bf[:nbf.value], e2q, node, len(e))


def plane_data(khat=(1.0, 0.0, 0.0), kmag=2 * np.pi, pol=(0.0, 1.0, 0.0), amp=1.0, phase=0.0):
    d = Data()
    d.kind = DATA_PLANE
    d.khat[:] = [float(v) for v in khat]
    d.kmag = float(kmag)
    d.pol[:] = [float(v) for v in pol]
    d.amp = float(amp)
    d.phase = float(phase)
    return d


def cavity_data():
    d = Data()
    d.kind = DATA_CAVITY
    d.khat[:] = [1.0, 0.0, 0.0]
    d.pol[:] = [0.0, 1.0, 0.0]
    d.kmag = 0.0
    d.amp = 1.0
    d.phase = 0.0
    return d


def stationary_data():
    """maxwell_imposed_stationary (src/models/maxwell.c:16-84)."""
    d = cavity_data()
    d.kind = DATA_STATIONARY
    return d


def eval_data(data: Data, xyz: np.ndarray, t: float, device: int = 0) -> np.ndarray:
    """The analytic data at points xyz[n, 3] and time t, evaluated on the
    device by the solver's own code: [n, 6]."""
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    w = np.zeros((len(x), 6))
    check(lib().gdn_cuda_eval_data(C.byref(data), len(x), _dp(x), float(t), _dp(w), device))
    return w


class Solver:
    """One attach handle (the device-side replacement of a gdn_simulation's
    assembled operators)."""

    def __init__(self, mesh: MeshArrays, scheme=SCHEME_RK3, data: Data = None, dt: float = None,
                 precision=FP64, nb_v=4, tables: Tables = None, device=0, use_graph=1,
                 refine_passes=1, theta=0.5, rk3_variant=0, kin_sweep=0, boundary_flux=BC_UPWIND):
        self.L = lib()
        self.h = C.c_void_p()
        self.mesh = mesh
        self.scheme = scheme
        self.tables = tables if tables is not None else t10_tables()
        self.data = data if data is not None else plane_data()
        model = self._model(scheme, nb_v, theta, boundary_flux)
        cfg = Config(precision, refine_passes, rk3_variant, use_graph, device, kin_sweep)
        check(self.L.gdn_cuda_attach(C.byref(mesh.struct), C.byref(self.tables), C.byref(model),
                                     C.byref(self.data), C.byref(cfg), float(dt), C.byref(self.h)))
        self.dt = float(dt)

    def _model(self, scheme, nb_v, theta, boundary_flux=BC_UPWIND):
        """The gdn_model descriptor of the scheme (vi kept alive on self)."""
        if scheme == SCHEME_RK3:
            self._vi = np.zeros(3, np.float64)
            self.m = 6
            model = Model(SCHEME_RK3, 6, 0, 1.0, 0.0, _dp(self._vi), 0.5, boundary_flux)
        else:
            lam = D3Q4_LAMBDA if nb_v == 4 else D3Q6_LAMBDA
            base = D3Q4_VI if nb_v == 4 else D3Q6_VI
            self._vi = np.ascontiguousarray((base * lam).ravel())
            self.m = 6 * nb_v
            model = Model(SCHEME_KINETIC, 6, nb_v, lam, RELAX_OMEGA, _dp(self._vi), theta, boundary_flux)
        self.nb_v = nb_v
        self._model_struct = model
        return model

    @property
    def wlen(self) -> int:
        n = C.c_longlong()
        check(self.L.gdn_cuda_state_size(self.h, C.byref(n)))
        return n.value

    def solve(self, itermax: int):
        wn = np.zeros(self.wlen, np.float64)
        t, cpu = C.c_double(), C.c_double()
        check(self.L.gdn_cuda_solve(self.h, int(itermax), _dp(wn), C.byref(t), C.byref(cpu)))
        return wn, t.value, cpu.value

    def init(self):
        check(self.L.gdn_cuda_init(self.h))

    def advance(self, n: int):
        check(self.L.gdn_cuda_advance(self.h, int(n)))

    def set_state(self, wn: np.ndarray, t: float):
        w = np.ascontiguousarray(wn, dtype=np.float64)
        check(self.L.gdn_cuda_set_state(self.h, _dp(w), float(t)))

    def get_state(self) -> np.ndarray:
        wn = np.zeros(self.wlen, np.float64)
        check(self.L.gdn_cuda_get_state(self.h, _dp(wn)))
        return wn

    def step_host(self, wn: np.ndarray, n: int):
        assert wn.dtype == np.float64 and wn.flags.c_contiguous
        check(self.L.gdn_cuda_step_host(self.h, _dp(wn), int(n)))

    def save_xdmf(self, basename: str, iter_id: int, instance: int = 0):
        """io_save_all of the current state (raw binary + XDMF files)."""
        check(self.L.gdn_cuda_save_xdmf(self.h, int(instance), basename.encode(), int(iter_id)))

    def set_wait_limit(self, polls: int):
        """Polls after which a bounded device-side wait gives up (test hook)."""
        check(self.L.gdn_cuda_set_wait_limit(self.h, int(polls)))

    def error_l2(self) -> float:
        e = C.c_double()
        check(self.L.gdn_cuda_error_l2(self.h, C.byref(e)))
        return e.value

    @property
    def t(self) -> float:
        t = C.c_double()
        check(self.L.gdn_cuda_get_time(self.h, C.byref(t)))
        return t.value

    @property
    def num_levels(self) -> int:
        n = C.c_int()
        check(self.L.gdn_cuda_num_levels(self.h, C.byref(n)))
        return n.value

    @property
    def kin_sweep_mode(self) -> int:
        n = C.c_int()
        check(self.L.gdn_cuda_kin_sweep_mode(self.h, C.byref(n)))
        return n.value

    @property
    def rk3_variant(self):
        """(variant in use, resident CTAs per SM it was compiled for)"""
        v, m = C.c_int(), C.c_int()
        check(self.L.gdn_cuda_rk3_variant(self.h, C.byref(v), C.byref(m)))
        return v.value, m.value

    @property
    def launches(self) -> int:
        n = C.c_longlong()
        check(self.L.gdn_cuda_launch_count(self.h, C.byref(n)))
        return n.value

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(self.L.gdn_cuda_stream(self.h, C.byref(s)))
        return s.value or 0

    def close(self):
        if self.h:
            self.L.gdn_cuda_detach(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver(Solver):
    """A batch of independent solves of one scheme in one handle
    (gdn_cuda_attach_batch): every stage / step launch covers all instances;
    each instance keeps its own mesh, data and dt."""

    def __init__(self, meshes, datas, dts, scheme=SCHEME_RK3, precision=FP64, nb_v=4, tables: Tables = None,
                 device=0, use_graph=1, refine_passes=1, theta=0.5, rk3_variant=0, kin_sweep=0):
        self.L = lib()
        self.h = C.c_void_p()
        self.meshes = list(meshes)
        self.datas = list(datas)
        self.scheme = scheme
        self.tables = tables if tables is not None else t10_tables()
        model = self._model(scheme, nb_v, theta)
        n = len(self.meshes)
        self._inst = (Instance * n)()
        for i in range(n):
            self._inst[i].mesh = C.pointer(self.meshes[i].struct)
            self._inst[i].model = C.pointer(model)
            self._inst[i].data = C.pointer(self.datas[i])
            self._inst[i].dt = float(dts[i])
        cfg = Config(precision, refine_passes, rk3_variant, use_graph, device, kin_sweep)
        check(self.L.gdn_cuda_attach_batch(self._inst, n, C.byref(self.tables), C.byref(cfg), C.byref(self.h)))
        self.dts = [float(d) for d in dts]
        self.dt = self.dts[0]

    @property
    def ninst(self) -> int:
        n = C.c_int()
        check(self.L.gdn_cuda_num_instances(self.h, C.byref(n)))
        return n.value

    def instance_info(self, i: int):
        """(t, nbelems, offset, length) of instance i in the batch state."""
        t, ne, off, ln = C.c_double(), C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(self.L.gdn_cuda_instance_info(self.h, int(i), C.byref(t), C.byref(ne), C.byref(off), C.byref(ln)))
        return t.value, ne.value, off.value, ln.value

    def split(self, wn: np.ndarray):
        """The batch state as a list of per-instance reference-layout views."""
        out = []
        for i in range(self.ninst):
            _, _, off, ln = self.instance_info(i)
            out.append(wn[off:off + ln])
        return out

    def error_l2_batch(self) -> np.ndarray:
        e = np.zeros(self.ninst, np.float64)
        check(self.L.gdn_cuda_error_l2_batch(self.h, _dp(e)))
        return e


def _conv_model(scheme, nb_v, boundary_flux):
    holder = Solver.__new__(Solver)
    model = Solver._model(holder, scheme, nb_v, 0.5, boundary_flux)
    return holder, model


def time_convergence(mesh: MeshArrays, scheme, data, init_dt: float, tmax: float, nb_run: int,
                     precision=FP64, nb_v=4, boundary_flux=BC_UPWIND, tables: Tables = None, device=0):
    """utils_l2_time_convergence on the device (gdn_cuda_time_convergence):
    returns dict(dt, iter, err, order) arrays over the dt-halving runs."""
    L = lib()
    tabs = tables if tables is not None else t10_tables()
    holder, model = _conv_model(scheme, nb_v, boundary_flux)
    cfg = Config(precision, 1, 0, 1, device, 0)
    dt, err, order = (np.zeros(nb_run) for _ in range(3))
    it = np.zeros(nb_run, np.int32)
    check(L.gdn_cuda_time_convergence(C.byref(mesh.struct), C.byref(tabs), C.byref(model), C.byref(data),
                                      C.byref(cfg), float(init_dt), float(tmax), int(nb_run), _dp(dt), _ip(it),
                                      _dp(err), _dp(order)))
    return dict(dt=dt, iter=it, err=err, order=order)


def space_convergence(meshes, scheme, data, init_dt: float, tmax: float, time_refinement=True, precision=FP64,
                      nb_v=4, boundary_flux=BC_UPWIND, tables: Tables = None, device=0):
    """utils_l2_space_convergence on the device (gdn_cuda_space_convergence):
    returns dict(dt, iter, hmin, err, order) over the meshes."""
    L = lib()
    tabs = tables if tables is not None else t10_tables()
    holder, model = _conv_model(scheme, nb_v, boundary_flux)
    cfg = Config(precision, 1, 0, 1, device, 0)
    n = len(meshes)
    ptrs = (C.POINTER(Mesh) * n)(*[C.pointer(m.struct) for m in meshes])
    dt, hmin, err, order = (np.zeros(n) for _ in range(4))
    it = np.zeros(n, np.int32)
    check(L.gdn_cuda_space_convergence(ptrs, n, C.byref(tabs), C.byref(model), C.byref(data), C.byref(cfg),
                                       float(init_dt), float(tmax), int(bool(time_refinement)), _dp(dt), _ip(it),
                                       _dp(hmin), _dp(err), _dp(order)))
    return dict(dt=dt, iter=it, hmin=hmin, err=err, order=order)
