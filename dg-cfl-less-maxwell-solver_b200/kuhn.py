"""Seeded synthetic meshes: the unit cube cut into n^3 cubes, each cube into the
6 Kuhn tetrahedra, with optional uniform jitter of the interior vertices.

The reference reads gmsh v2.2 ASCII T4 meshes (src/mesh/mesh.c:623-726) and
requires nodes/elements numbered 1..N (asserts at mesh.c:484, :545) and every
tetrahedron positively oriented (the Heron/Jacobian checks at mesh.c:194-195
fail otherwise).  `write_msh22` writes exactly that format with %.17g
coordinates so that the reference's atof parse reproduces the doubles bit for
bit.

Jitter: interior vertex v, component c, attempt a draws
u = splitmix64(splitmix64(seed) + 4 v + c + (a << 40)) / 2^64 and moves by
J h (2u - 1).  Vertices of a tetrahedron whose Jacobian determinant would fall
below 5% of the unjittered value are redrawn with the next attempt number.
"""
from __future__ import annotations

import itertools

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """Vectorised splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = (np.asarray(x, dtype=np.uint64) + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counter: np.ndarray) -> np.ndarray:
    """Counter-based uniform [0, 1) doubles from the top 53 bits."""
    base = splitmix64(np.array([seed & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        z = splitmix64(base + np.asarray(counter, dtype=np.uint64))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _tet_det(p: np.ndarray, tets: np.ndarray) -> np.ndarray:
    a = p[tets[:, 1]] - p[tets[:, 0]]
    b = p[tets[:, 2]] - p[tets[:, 0]]
    c = p[tets[:, 3]] - p[tets[:, 0]]
    return np.einsum("ij,ij->i", a, np.cross(b, c))


def kuhn_cube(n: int, jitter: float = 0.0, seed: int = 0):
    """Returns (coords[nv,3] float64, elem2node[ne,4] int32, 0-based).

    Element order: cube (i, j, k) with i fastest, then the 6 Kuhn tets of the
    cube for the permutations of (x, y, z) in lexicographic order.  Each tet is
    (v000, v000 + e_a, v000 + e_a + e_b, v111) with vertices 1 and 2 swapped
    when that ordering has a negative Jacobian.
    """
    if n < 1:
        raise ValueError("n must be >= 1")
    h = 1.0 / n
    m = n + 1
    ii, jj, kk = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    # vertex index v = i + m (j + m k)
    vi = ii.transpose(2, 1, 0).ravel()
    vj = jj.transpose(2, 1, 0).ravel()
    vk = kk.transpose(2, 1, 0).ravel()
    base = np.stack([vi, vj, vk], axis=1).astype(np.float64) * h
    # exact endpoints: the boundary planes stay at 0 and 1
    base[vi == n, 0] = 1.0
    base[vj == n, 1] = 1.0
    base[vk == n, 2] = 1.0

    cube = np.arange(n ** 3)
    ci = cube % n
    cj = (cube // n) % n
    ck = cube // (n * n)
    v000 = ci + m * (cj + m * ck)
    step = np.array([1, m, m * m])
    tets = []
    for perm in itertools.permutations(range(3)):
        a, b, _ = perm
        t = np.stack([v000, v000 + step[a], v000 + step[a] + step[b],
                      v000 + step.sum()], axis=1)
        tets.append(t)
    tets = np.stack(tets, axis=1).reshape(-1, 4)
    d = _tet_det(base, tets)
    neg = d < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    det0 = np.abs(d)

    coords = base.copy()
    if jitter > 0.0:
        interior = (vi > 0) & (vi < n) & (vj > 0) & (vj < n) & (vk > 0) & (vk < n)
        idx = np.nonzero(interior)[0].astype(np.uint64)
        attempt = np.zeros(len(base), dtype=np.uint64)
        for _ in range(64):
            cnt = (idx[:, None] * np.uint64(4) + np.arange(3, dtype=np.uint64)[None, :]
                   + (attempt[idx][:, None] << np.uint64(40)))
            u = uniform01(seed, cnt)
            coords = base.copy()
            coords[idx.astype(np.int64)] += jitter * h * (2.0 * u - 1.0)
            dj = _tet_det(coords, tets)
            bad = dj < 0.05 * det0
            if not bad.any():
                break
            badv = np.unique(tets[bad].ravel())
            badv = badv[interior[badv]]
            attempt[badv] += np.uint64(1)
        else:  # pragma: no cover - would need an absurd jitter
            raise RuntimeError("jittered Kuhn mesh could not be made valid")
    return coords, tets.astype(np.int32)


def random_plane_wave(seed: int, kmag: float):
    """Random unit direction (normalised Gaussian triple), polarisation
    orthogonal to it, for the plane-wave configurations."""
    rng = np.random.Generator(np.random.Philox(seed))
    k = rng.standard_normal(3)
    k /= np.linalg.norm(k)
    q = rng.standard_normal(3)
    p = q - np.dot(q, k) * k
    p /= np.linalg.norm(p)
    return k, float(kmag), p


def uneven_plane_wave_batch(seed: int, count: int, n_lo: int = 8, n_hi: int = 40, jitter: float = 0.1,
                            kmag_lo: float = 2 * np.pi, kmag_hi: float = 8 * np.pi):
    """Specs of `count` independent plane-wave solves of uneven size.

    Instance i draws everything from z_i = splitmix64(seed + i): the cube
    resolution n uniform in [n_lo, n_hi], the jitter seed z_i (jitter +/-J h),
    and, from a Philox generator keyed by z_i, a unit wave direction (a
    normalised Gaussian triple), |k| uniform in [kmag_lo, kmag_hi] and a
    polarisation orthogonal to the direction.  Even i run RK3, odd i the
    CFL-less scheme.  Returns a list of dicts.
    """
    out = []
    z = splitmix64(np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.arange(count, dtype=np.uint64))
    for i in range(count):
        zi = int(z[i])
        n = n_lo + zi % (n_hi - n_lo + 1)
        rng = np.random.Generator(np.random.Philox(zi))
        k = rng.standard_normal(3)
        k /= np.linalg.norm(k)
        kmag = kmag_lo + (kmag_hi - kmag_lo) * rng.random()
        q = rng.standard_normal(3)
        p = q - np.dot(q, k) * k
        p /= np.linalg.norm(p)
        out.append({"index": i, "n": int(n), "jitter": jitter, "jitter_seed": zi, "khat": k, "kmag": float(kmag),
                    "pol": p, "scheme": "rk3" if i % 2 == 0 else "kinetic"})
    return out


def write_msh22(path: str, coords: np.ndarray, elem2node: np.ndarray) -> None:
    """gmsh v2.2 ASCII, 1-based, type-4 elements with two tags."""
    nv = len(coords)
    ne = len(elem2node)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % nv)
        for i in range(nv):
            x, y, z = coords[i]
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, x, y, z))
        f.write("$EndNodes\n$Elements\n%d\n" % ne)
        for e in range(ne):
            a, b, c, d = (int(v) + 1 for v in elem2node[e])
            f.write("%d 4 2 1 1 %d %d %d %d\n" % (e + 1, a, b, c, d))
        f.write("$EndElements\n")


def read_msh22(path: str):
    """Reads a gmsh 2.2 ASCII file; returns (coords, elem2node 0-based) with
    only the type-4 (T4) elements, in file order (what mesh.c:506-621 keeps)."""
    with open(path) as f:
        lines = f.read().split("\n")
    i = lines.index("$Nodes")
    nv = int(lines[i + 1])
    coords = np.array([[float(t) for t in lines[i + 2 + k].split()[1:4]]
                       for k in range(nv)])
    j = lines.index("$Elements")
    ne_all = int(lines[j + 1])
    tets = []
    for k in range(ne_all):
        tok = lines[j + 2 + k].split()
        if int(tok[1]) == 4:
            ntag = int(tok[2])
            tets.append([int(t) - 1 for t in tok[3 + ntag:7 + ntag]])
    return coords, np.array(tets, dtype=np.int32)
