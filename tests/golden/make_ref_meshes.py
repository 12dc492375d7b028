"""Makes tests/golden/ref_meshes.npz: the three gmsh meshes the reference ships
(data/mesh/t4_cube_8.msh, t4_cube_16.msh, t4_cube_8_torus_128.msh), as the
reference's own reader (mesh_read_from_msh22_file, src/mesh/mesh.c:623-726,
compiled in place into oracle/_ref) leaves them: vertex coordinates and the
T4 element list, 0-based.  Arrays only; the tests write them back as msh22
files (gdon3d_b200.kuhn.write_msh22, %.17g coordinates) and read those through
the reference's reader again.

Before saving, each mesh is checked to round-trip: the re-written file gives
the reader the same vertices and elements bit for bit, and the reference's
mesh_build_connectivity the same face2elem, fnode2enode, boundaryface,
elem2qnode and P2 nodes as the original file.

Run here, where the reference tree exists:
    python tests/golden/make_ref_meshes.py [reference_tree]
(default: $GDN_REFERENCE_TREE, else a checkout named "reference" beside this
repository).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import conftest  # noqa: E402,F401  (loads the package as gdon3d_b200)
from gdon3d_b200 import kuhn  # noqa: E402
from oracle import ref  # noqa: E402

NAMES = ["t4_cube_8", "t4_cube_16", "t4_cube_8_torus_128"]


def main():
    tree = (sys.argv[1] if len(sys.argv) > 1 else None) or os.environ.get("GDN_REFERENCE_TREE") or \
        os.path.join(os.path.dirname(ROOT), "reference")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name in NAMES:
            src = os.path.join(tree, "data", "mesh", name + ".msh")
            coords, e2n = ref.msh_read_raw(src)
            again = os.path.join(tmp, name + ".msh")
            kuhn.write_msh22(again, coords, e2n)
            c2, e2 = ref.msh_read_raw(again)
            assert np.array_equal(c2, coords) and np.array_equal(e2, e2n), name
            a0 = ref.RefMesh(path=src).arrays()
            a1 = ref.RefMesh(path=again).arrays()
            for k in a0:
                assert np.array_equal(a0[k], a1[k]), (name, k)
            out[name + "_coords"] = coords
            out[name + "_elem2node"] = e2n.astype(np.int32)
            print("%s: %d vertices, %d tetrahedra, round trip exact" % (name, len(coords), len(e2n)))
    np.savez_compressed(os.path.join(HERE, "ref_meshes.npz"), **out)


if __name__ == "__main__":
    main()
