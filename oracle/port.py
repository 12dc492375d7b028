"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

ctypes access to oracle/_build/libgdon3d_oracle.so, the repo's CPU
restatement (gdn_oracle.c) of the RK3 and CFL-less hot paths.  It takes the
reference's mesh arrays and P2 tables and returns states in the reference's
wn layout.  Used by tests/ as the checker and by bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libgdon3d_oracle.so")


class OrcMesh(C.Structure):
    _fields_ = [("nbelems", C.c_int), ("nbfaces", C.c_int), ("nboundaryfaces", C.c_int),
                ("nbqnodes", C.c_int), ("face2elem", C.POINTER(C.c_int)),
                ("fnode2enode", C.POINTER(C.c_int)), ("boundaryface", C.POINTER(C.c_int)),
                ("elem2qnode", C.POINTER(C.c_int)), ("node", C.POINTER(C.c_double))]


class OrcTables(C.Structure):
    _fields_ = [("wpg", C.c_double * 10), ("mass", (C.c_double * 10) * 10),
                ("inv_mass", (C.c_double * 10) * 10), ("internal", ((C.c_double * 3) * 10) * 10),
                ("face_scal", (C.c_double * 6) * 6), ("ref_normal", (C.c_double * 3) * 4),
                ("face2node", (C.c_int * 6) * 4)]


class OrcData(C.Structure):
    _fields_ = [("kind", C.c_int), ("khat", C.c_double * 3), ("kmag", C.c_double),
                ("pol", C.c_double * 3), ("amp", C.c_double), ("phase", C.c_double)]


class OrcKin(C.Structure):
    _fields_ = [("nb_v", C.c_int), ("vi", C.c_double * 18), ("lambda_", C.c_double),
                ("omega", C.c_double), ("theta", C.c_double)]


D3Q4_LAMBDA = 1.732050807568877293
D3Q4_VI = [[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]]
D3Q6_LAMBDA = 3.0
D3Q6_VI = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]]

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        L.orc_rk3_run.restype = C.c_int
        L.orc_rk3_run.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcTables), C.POINTER(OrcData),
                                  C.c_double, C.c_int, dp, dp]
        L.orc_kin_run.restype = C.c_int
        L.orc_kin_run.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcTables), C.POINTER(OrcData),
                                  C.POINTER(OrcKin), C.c_double, C.c_int, dp, dp]
        L.orc_error_l2.restype = C.c_double
        L.orc_error_l2.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcTables), C.POINTER(OrcData),
                                   C.c_int, dp, C.c_double]
        _lib = L
    return _lib


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """Holds the mesh arrays (dict with face2elem, fnode2enode, boundaryface,
    elem2qnode, node as numpy arrays), the tables (dict) and the data."""

    def __init__(self, nbelems, arrays: dict, tables: dict):
        self.a = {k: np.ascontiguousarray(v, dtype=np.float64 if k == "node" else np.int32)
                  for k, v in arrays.items()}
        bf = self.a["boundaryface"] if len(self.a["boundaryface"]) else np.zeros(1, np.int32)
        self._bf = bf
        self.nbelems = int(nbelems)
        self.nbf = len(self.a["boundaryface"])
        self.neq = 10 * self.nbelems + 6 * self.nbf
        self.m = OrcMesh(self.nbelems, len(self.a["face2elem"]) // 4, self.nbf,
                         len(self.a["node"]) // 3, _ip(self.a["face2elem"]),
                         _ip(self.a["fnode2enode"]), _ip(bf), _ip(self.a["elem2qnode"]),
                         _dp(self.a["node"]))
        self.t = OrcTables()
        for k in ("wpg", "mass", "inv_mass", "internal", "face_scal", "ref_normal", "face2node"):
            np.ctypeslib.as_array(getattr(self.t, k))[:] = np.asarray(tables[k])

    @staticmethod
    def data(kind=0, khat=(1, 0, 0), kmag=2 * np.pi, pol=(0, 1, 0), amp=1.0, phase=0.0):
        d = OrcData()
        d.kind = kind
        d.khat[:] = [float(x) for x in khat]
        d.kmag = float(kmag)
        d.pol[:] = [float(x) for x in pol]
        d.amp = float(amp)
        d.phase = float(phase)
        return d

    def rk3(self, data: OrcData, dt: float, steps: int):
        wn = np.zeros(6 * self.neq)
        t = C.c_double()
        rc = lib().orc_rk3_run(C.byref(self.m), C.byref(self.t), C.byref(data), dt, steps,
                               _dp(wn), C.byref(t))
        assert rc == 0
        return wn, t.value

    def kinetic(self, data: OrcData, dt: float, steps: int, nb_v=4, theta=0.5,
                omega=1.999999999999):
        k = OrcKin()
        k.nb_v = nb_v
        lam = D3Q4_LAMBDA if nb_v == 4 else D3Q6_LAMBDA
        vi = np.array(D3Q4_VI if nb_v == 4 else D3Q6_VI, dtype=np.float64) * lam
        np.ctypeslib.as_array(k.vi)[: 3 * nb_v] = vi.ravel()
        k.lambda_ = lam
        k.omega = omega
        k.theta = theta
        wn = np.zeros(6 * nb_v * self.neq)
        t = C.c_double()
        rc = lib().orc_kin_run(C.byref(self.m), C.byref(self.t), C.byref(data), C.byref(k), dt,
                               steps, _dp(wn), C.byref(t))
        if rc != 0:
            raise RuntimeError("oracle kinetic run failed (%d)" % rc)
        return wn, t.value

    def error_l2(self, data: OrcData, wn: np.ndarray, t: float, nb_v=0) -> float:
        w = np.ascontiguousarray(wn, dtype=np.float64)
        return float(lib().orc_error_l2(C.byref(self.m), C.byref(self.t), C.byref(data), nb_v,
                                        _dp(w), t))
