"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

ctypes access to oracle/_ref/libgdon3d_ref_{zero,pattern}.so: the reference's
own C sources (src/mesh, src/models, src/simulation, src/dg) compiled in place
by oracle/Makefile against the repo-owned sparse shim, driven by
oracle/ref_driver.c.  Only tests, __graft_entry__.smoke() and the CPU-baseline
legs of bench.py use this module, and only as a checker / timed baseline.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

SCHEME_RK3, SCHEME_D3Q4, SCHEME_D3Q6 = 0, 1, 2
SCHEME_RK3_METAL = 3  # RK3 with the metal boundary flux (maxwell.c:205-223)
# analytic data of ref_driver.c: the plane wave, the reference's cavity and
# stationary data, the examples' cos wave (examples/rk3_maxwell_plane_wave.c:35-47)
DATA_PLANE, DATA_CAVITY, DATA_STATIONARY, DATA_EXAMPLE_COS = 0, 1, 2, 3


class RefData(C.Structure):
    _fields_ = [("kind", C.c_int), ("khat", C.c_double * 3), ("kmag", C.c_double),
                ("pol", C.c_double * 3), ("amp", C.c_double), ("phase", C.c_double)]


def make_data(kind=DATA_PLANE, khat=(1.0, 0.0, 0.0), kmag=2 * np.pi,
              pol=(0.0, 1.0, 0.0), amp=1.0, phase=0.0) -> RefData:
    d = RefData()
    d.kind = kind
    d.khat[:] = [float(v) for v in khat]
    d.kmag = float(kmag)
    d.pol[:] = [float(v) for v in pol]
    d.amp = float(amp)
    d.phase = float(phase)
    return d


_libs: dict = {}
_libc = C.CDLL(None)


class _stdout_to_stderr:
    """The reference prints progress to stdout (explicit.c:98-101,
    relaxation.c:167-170); keep the caller's stdout clean by sending C stdout
    to stderr while reference code runs."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        _libc.fflush(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        _libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


def available(variant: str = "zero") -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libgdon3d_ref_%s.so" % variant))


def lib(variant: str = "zero"):
    if variant in _libs:
        return _libs[variant]
    path = os.path.join(REF_DIR, "libgdon3d_ref_%s.so" % variant)
    L = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.ref_mesh_from_file.restype = vp
    L.ref_mesh_from_file.argtypes = [C.c_char_p]
    L.ref_mesh_from_arrays.restype = vp
    L.ref_mesh_from_arrays.argtypes = [C.c_int, dp, C.c_int, ip]
    L.ref_mesh_info.argtypes = [vp, ip]
    L.ref_mesh_arrays.argtypes = [vp, ip, ip, ip, ip, dp]
    L.ref_mesh_hmin.restype = C.c_double
    L.ref_mesh_hmin.argtypes = [vp]
    L.ref_mesh_free.argtypes = [vp]
    L.ref_wlen.restype = C.c_int
    L.ref_wlen.argtypes = [vp, C.c_int]
    L.ref_run.restype = C.c_int
    L.ref_run.argtypes = [vp, C.c_int, C.POINTER(RefData), C.c_double, C.c_int,
                          dp, dp, dp, dp, dp]
    L.ref_error_l2.restype = C.c_double
    L.ref_error_l2.argtypes = [vp, C.c_int, C.POINTER(RefData), dp, C.c_double]
    L.ref_init_state.argtypes = [vp, C.c_int, C.POINTER(RefData), dp]
    L.ref_t10_tables.argtypes = [dp, dp, dp, dp, dp, dp, ip]
    L.ref_msh_read_raw.argtypes = [C.c_char_p, ip, ip, dp, ip]
    L.ref_eval_data.argtypes = [C.POINTER(RefData), C.c_int, dp, C.c_double, dp]
    L.ref_time_convergence.restype = C.c_int
    L.ref_time_convergence.argtypes = [C.c_char_p, C.c_int, C.POINTER(RefData), C.c_double, C.c_double,
                                       C.c_int, C.c_int, vp]
    if variant == "bound":
        L.ref_run_bound.restype = C.c_int
        L.ref_run_bound.argtypes = [vp, C.c_int, C.POINTER(RefData), vp, C.c_int, C.c_double, C.c_int,
                                    dp, dp, dp, dp]
        L.ref_bound_message.restype = C.c_char_p
    _libs[variant] = L
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class RefMesh:
    """A gdn_mesh built by the reference's reader/connectivity builder."""

    def __init__(self, coords=None, elem2node=None, path=None, variant="zero"):
        self.L = lib(variant)
        if path is not None:
            with _stdout_to_stderr():
                self.h = self.L.ref_mesh_from_file(path.encode())
        else:
            c = np.ascontiguousarray(coords, dtype=np.float64)
            e = np.ascontiguousarray(elem2node, dtype=np.int32)
            self.h = self.L.ref_mesh_from_arrays(len(c), _dp(c), len(e), _ip(e))
        info = np.zeros(4, dtype=np.int32)
        self.L.ref_mesh_info(self.h, _ip(info))
        self.nbelems, self.nbfaces, self.nboundaryfaces, self.nbqnodes = map(int, info)

    def arrays(self):
        ne, nf, nb, nq = self.nbelems, self.nbfaces, self.nboundaryfaces, self.nbqnodes
        f2e = np.zeros(4 * nf, np.int32)
        fn = np.zeros(12 * nf, np.int32)
        bf = np.zeros(max(nb, 1), np.int32)
        e2q = np.zeros(10 * ne + 6 * nb, np.int32)
        node = np.zeros(3 * nq, np.float64)
        self.L.ref_mesh_arrays(self.h, _ip(f2e), _ip(fn), _ip(bf), _ip(e2q), _dp(node))
        return dict(face2elem=f2e, fnode2enode=fn, boundaryface=bf[:nb],
                    elem2qnode=e2q, node=node)

    def hmin(self) -> float:
        return float(self.L.ref_mesh_hmin(self.h))

    def neq(self) -> int:
        return 10 * self.nbelems + 6 * self.nboundaryfaces

    def run(self, scheme, data: RefData, dt: float, steps: int):
        """dg_solve through the reference; returns dict(wn, t, err, cpu_run, cpu_asm)."""
        wlen = self.L.ref_wlen(self.h, scheme)
        wn = np.zeros(wlen, np.float64)
        t, err, crun, casm = (C.c_double() for _ in range(4))
        with _stdout_to_stderr():
            rc = self.L.ref_run(self.h, scheme, C.byref(data), dt, steps, _dp(wn),
                                C.byref(t), C.byref(err), C.byref(crun), C.byref(casm))
        if rc != 0:
            raise RuntimeError("reference run did not produce %d steps" % steps)
        return dict(wn=wn, t=t.value, err=err.value, cpu_run=crun.value,
                    cpu_asm=casm.value)

    def run_bound(self, scheme, data: RefData, gpu_data, dt: float, steps: int, precision: int = 0):
        """The reference's flow through the product's binding (variant
        "bound" only): simulation_init, simulation_set_time_parameters,
        dg_cuda_attach(gpu_data: a gdon3d_cuda gdn_cuda_data), dg_solve routed
        to the GPU, simulation_error_l2.  Returns dict(rc, msg, wn, t, err,
        mismatch)."""
        wlen = self.L.ref_wlen(self.h, scheme)
        wn = np.zeros(wlen, np.float64)
        t, err, mis = (C.c_double() for _ in range(3))
        with _stdout_to_stderr():
            rc = self.L.ref_run_bound(self.h, scheme, C.byref(data), C.cast(C.byref(gpu_data), C.c_void_p),
                                      precision, dt, steps, _dp(wn), C.byref(t), C.byref(err), C.byref(mis))
        return dict(rc=rc, msg=self.L.ref_bound_message().decode(), wn=wn, t=t.value, err=err.value,
                    mismatch=mis.value)

    def error_l2(self, scheme, data: RefData, wn: np.ndarray, t: float) -> float:
        w = np.ascontiguousarray(wn, dtype=np.float64)
        return float(self.L.ref_error_l2(self.h, scheme, C.byref(data), _dp(w), t))

    def init_state(self, scheme, data: RefData) -> np.ndarray:
        wn = np.zeros(self.L.ref_wlen(self.h, scheme), np.float64)
        self.L.ref_init_state(self.h, scheme, C.byref(data), _dp(wn))
        return wn

    def close(self):
        if self.h:
            self.L.ref_mesh_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_convergence(path: str, scheme: int, data: RefData, init_dt: float, tmax: float, nb_run: int,
                     variant: str = "zero", gpu_data=None):
    """The reference's utils_l2_time_convergence on a msh file; with
    variant "bound" and gpu_data, every dg_solve routed to the GPU through the
    binding.  Returns the per-run rows it printed: dict(dt, iter, error, order)
    (order None for the first run)."""
    import re
    import tempfile
    L = lib(variant)
    with tempfile.TemporaryFile(mode="w+") as out:
        import sys
        sys.stdout.flush()
        _libc.fflush(None)
        saved = os.dup(1)
        os.dup2(out.fileno(), 1)
        try:
            rc = L.ref_time_convergence(path.encode(), scheme, C.byref(data), init_dt, tmax, nb_run,
                                        1 if gpu_data is not None else 0,
                                        C.cast(C.byref(gpu_data), C.c_void_p) if gpu_data is not None else None)
        finally:
            _libc.fflush(None)
            os.dup2(saved, 1)
            os.close(saved)
        out.seek(0)
        text = out.read()
    if rc != 0:
        raise RuntimeError("reference convergence driver: status %d" % rc)
    rows = []
    for line in re.split(r"[\r\n]+", text):
        f = line.split()
        if len(f) == 12 and f[0] == "fooo":
            rows.append(dict(dt=float(f[6]), iter=int(f[3]), error=float(f[10]),
                             order=None if f[11] == "---" else float(f[11])))
    return rows


def eval_callback(kind: int, xyz: np.ndarray, t: float, variant: str = "zero", **kw) -> np.ndarray:
    """The reference-side callback of data `kind` (ref_driver.c select_data)
    at points xyz[n, 3] and time t: [n, 6]."""
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    w = np.zeros((len(x), 6))
    lib(variant).ref_eval_data(C.byref(make_data(kind=kind, **kw)), len(x), _dp(x), float(t), _dp(w))
    return w


def msh_read_raw(path: str, variant: str = "zero"):
    """(coords[n, 3], elem2node[ne, 4] 0-based) of a msh22 file as the
    reference's reader leaves them (T4 elements only, no connectivity)."""
    L = lib(variant)
    nn, ne = C.c_int(), C.c_int()
    with _stdout_to_stderr():
        L.ref_msh_read_raw(path.encode(), C.byref(nn), C.byref(ne), None, None)
        coords = np.zeros((nn.value, 3))
        e2n = np.zeros((ne.value, 4), np.int32)
        L.ref_msh_read_raw(path.encode(), C.byref(nn), C.byref(ne), _dp(coords), _ip(e2n))
    return coords, e2n


def t10_tables(variant: str = "zero"):
    L = lib(variant)
    wpg = np.zeros(10)
    mass = np.zeros(100)
    inv = np.zeros(100)
    internal = np.zeros(300)
    fs = np.zeros(36)
    rn = np.zeros(12)
    f2n = np.zeros(24, np.int32)
    L.ref_t10_tables(_dp(wpg), _dp(mass), _dp(inv), _dp(internal), _dp(fs), _dp(rn), _ip(f2n))
    return dict(wpg=wpg, mass=mass.reshape(10, 10), inv_mass=inv.reshape(10, 10),
                internal=internal.reshape(10, 10, 3), face_scal=fs.reshape(6, 6),
                ref_normal=rn.reshape(4, 3), face2node=f2n.reshape(4, 6))
