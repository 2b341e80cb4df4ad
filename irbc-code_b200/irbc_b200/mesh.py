"""Membrane meshes: the reference's V/E/T text format and the discocyte
generator for the large workload.

File format (read by maincode.cpp:174-272): the vertex file holds one
`x y z` line per vertex, the edge file one `l1 l2` line per edge and the
triangle file one `t1 t2 t3` line per triangle, indices 1-based.  The
shipped trophozoite mesh orders triangle corners so that (B-A) x (C-A)
points outward and lists each edge once with l1 < l2; the generator keeps
both conventions.
"""
import os

import numpy as np

# Evans & Fung (1972) red-cell profile coefficients
EF_C0, EF_C1, EF_C2 = 0.207161, 2.002558, -1.122762


def icosphere(subdiv):
    """Unit icosphere after `subdiv` midpoint subdivisions:
    V = 10*4^n + 2, E = 30*4^n, F = 20*4^n."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    V = [np.array(v, float) / np.linalg.norm(v) for v in V]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        mid = {}

        def midpoint(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in mid:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                mid[key] = len(V) - 1
            return mid[key]
        nf = []
        for a, b, c in F:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = nf
    return np.array(V), np.array(F, np.int32)


def evans_fung(Vs, R):
    """Maps unit-sphere points onto the Evans-Fung discocyte of radius R:
    (x, y) scale by R; z = sign(z) R/2 sqrt(1-r^2) (C0 + C1 r^2 + C2 r^4),
    r^2 = x^2 + y^2 on the unit sphere."""
    x, y, z = Vs[:, 0], Vs[:, 1], Vs[:, 2]
    r2 = np.clip(x * x + y * y, 0.0, 1.0)
    h = 0.5 * R * np.sqrt(1.0 - r2) * (EF_C0 + EF_C1 * r2 + EF_C2 * r2 * r2)
    return np.stack([R * x, R * y, np.sign(z) * h], axis=1)


def edges_of(F):
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    e.sort(axis=1)
    e = np.unique(e, axis=0)
    return e.astype(np.int32)


def orient_outward(V, F):
    c = V.mean(axis=0)
    A, B, C = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    n = np.cross(B - A, C - A)
    flip = (((A + B + C) / 3.0 - c) * n).sum(axis=1) < 0
    F = F.copy()
    F[flip] = F[flip][:, [0, 2, 1]]
    return F


def discocyte(subdiv=4, R=4.0):
    """(V, E, T): 2562 vertices / 7680 edges / 5120 triangles for subdiv=4.
    Triangles are oriented on the sphere (where the test is exact) before
    the mapping, which preserves orientation."""
    Vs, F = icosphere(subdiv)
    F = orient_outward(Vs, F)
    V = evans_fung(Vs, R)
    return V, edges_of(F), F


def write_reference_files(folder, V, E, T, stem="Disc"):
    """Writes V/E/T in the reference's text format; returns the three paths."""
    os.makedirs(folder, exist_ok=True)
    n = len(V)
    pv = os.path.join(folder, "%sV%d.dat" % (stem, n))
    pe = os.path.join(folder, "%sE%d.dat" % (stem, n))
    pt = os.path.join(folder, "%sT%d.dat" % (stem, n))
    with open(pv, "w") as f:
        for x, y, z in V:
            f.write("%.9f\t%.9f\t%.9f\n" % (x, y, z))
    with open(pe, "w") as f:
        for a, b in E:
            f.write("%d\t%d\n" % (a + 1, b + 1))
    with open(pt, "w") as f:
        for a, b, c in T:
            f.write("%d\t%d\t%d\n" % (a + 1, b + 1, c + 1))
    return pv, pe, pt


def read_reference_files(pv, pe, pt):
    """Reads V/E/T files (1-based indices) -> V, 0-based E, T."""
    V = np.loadtxt(pv, dtype=np.float64).reshape(-1, 3)
    E = np.loadtxt(pe, dtype=np.int64).reshape(-1, 2) - 1
    T = np.loadtxt(pt, dtype=np.int64).reshape(-1, 3) - 1
    return V, E.astype(np.int32), T.astype(np.int32)


def discocyte_as_read(subdiv=4, R=4.0):
    """The discocyte exactly as a reader of the written files sees it
    (coordinates rounded to the file's 9 decimals)."""
    V, E, T = discocyte(subdiv, R)
    V = np.array([[float("%.9f" % c) for c in v] for v in V])
    return V, E, T
