"""Generates tests/golden/*.npz from the reference's own C code (oracle/_ref,
compiled in place from the reference sources by oracle/Makefile).

    python tests/golden/make_golden.py

Each fixture holds a seeded Kuhn mesh (coordinates, T4 connectivity), the
reference's connectivity arrays, the reference's P2 tables, and final states
of the reference's dg_solve for RK3 (plane wave), CFL-less d3q4 (PEC cavity)
and CFL-less d3q6 (plane wave).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dg-cfl-less-maxwell-solver_b200"))

import kuhn  # noqa: E402
from oracle import ref  # noqa: E402

CASES = [
    # name, n, jitter, seed, rk3 steps, d3q4 steps, d3q6 steps
    ("kuhn2", 2, 0.0, 1, 10, 5, 3),
    ("kuhn3j", 3, 0.15, 7, 12, 4, 0),
]
PLANE = dict(khat=(1.0, 0.0, 0.0), kmag=2 * np.pi, pol=(0.0, 1.0, 0.0))


def make(name, n, jitter, seed, s_rk3, s_q4, s_q6):
    c, e = kuhn.kuhn_cube(n, jitter, seed=seed)
    rm = ref.RefMesh(c, e)
    arrays = rm.arrays()
    hmin = rm.hmin()
    dt = 0.3 * hmin
    rk3 = rm.run(ref.SCHEME_RK3, ref.make_data(**PLANE), dt, s_rk3)
    q4 = rm.run(ref.SCHEME_D3Q4, ref.make_data(kind=ref.DATA_CAVITY), 10 * dt, s_q4)
    q6 = (rm.run(ref.SCHEME_D3Q6, ref.make_data(**PLANE), 10 * dt, s_q6) if s_q6
          else dict(wn=np.zeros(0), t=0.0, err=0.0))
    tabs = ref.t10_tables()
    out = dict(coords=c, elem2node=e, nbelems=rm.nbelems, hmin=hmin, dt=dt,
               rk3_steps=s_rk3, rk3_wn=rk3["wn"], rk3_t=rk3["t"], rk3_err=rk3["err"],
               q4_steps=s_q4, q4_wn=q4["wn"], q4_t=q4["t"], q4_err=q4["err"],
               q6_steps=s_q6, q6_wn=q6["wn"], q6_t=q6["t"], q6_err=q6["err"],
               plane=np.array(PLANE["khat"] + (PLANE["kmag"],) + PLANE["pol"]))
    for k, v in arrays.items():
        out["mesh_" + k] = v
    for k, v in tabs.items():
        out["t10_" + k] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, rm.nbelems, "tets; rk3 err %.6e, d3q4 err %.6e, d3q6 err %.6e"
          % (rk3["err"], q4["err"], q6["err"]))


if __name__ == "__main__":
    for case in CASES:
        make(*case)
