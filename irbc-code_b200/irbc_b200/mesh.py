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


def _pole_rotation(v):
    """rotation matrix taking the unit vector v to +z (Rodrigues)"""
    z = np.array([0.0, 0.0, 1.0])
    v = v / np.linalg.norm(v)
    ax = np.cross(v, z)
    s, c = np.linalg.norm(ax), float(v @ z)
    if s < 1e-15:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    ax /= s
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    return np.eye(3) + s * K + (1 - c) * (K @ K)


def _profile(theta, R):
    """Evans-Fung profile as a closed curve in the (r, z) half-plane,
    parameterised by the polar angle theta of the sphere point mapped there
    (evans_fung): r = R sin(theta), z = +-h(r)"""
    rho = np.sin(theta)
    r2 = rho * rho
    h = 0.5 * R * np.sqrt(np.clip(1.0 - r2, 0.0, 1.0)) * (EF_C0 + EF_C1 * r2 + EF_C2 * r2 * r2)
    return R * rho, np.where(theta <= 0.5 * np.pi, h, -h)


def _project(P, theta, R, newton=4, eps=1e-6):
    """Nearest points of the discocyte surface to the points P: each keeps
    its azimuth, and the profile parameter theta (started from its previous
    value) takes a few damped Newton steps on the squared (r, z) distance.
    Returns the surface points and their parameters."""
    rp, zp, phi = np.hypot(P[:, 0], P[:, 1]), P[:, 2], np.arctan2(P[:, 1], P[:, 0])
    for _ in range(newton):
        d = []
        for t in (theta - eps, theta, theta + eps):
            r, z = _profile(t, R)
            d.append((r - rp) ** 2 + (z - zp) ** 2)
        g = (d[2] - d[0]) / (2 * eps)
        hs = (d[2] - 2 * d[1] + d[0]) / (eps * eps)
        step = np.where(hs > 0, -g / np.maximum(hs, 1e-30), -np.sign(g) * 1e-3)
        theta = np.clip(theta + np.clip(step, -0.05, 0.05), 0.0, np.pi)
    r, z = _profile(theta, R)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1), theta


_cache = {}


def discocyte(subdiv=4, R=4.0, relax_iters=1000, step=0.2):
    """(V, E, T): 2562 vertices / 7680 edges / 5120 triangles for subdiv=4
    (fresh copies of a per-process cache; see _discocyte)."""
    key = (subdiv, R, relax_iters, step)
    if key not in _cache:
        _cache[key] = _discocyte(*key)
    return tuple(a.copy() for a in _cache[key])


def _discocyte(subdiv, R, relax_iters, step):
    """The discocyte mesh.

    The icosphere is turned so that one of its twelve 5-valent vertices sits
    on the axis (the others then lie at +-26.6 deg latitude, away from the
    rim), mapped onto the Evans-Fung surface (evans_fung), and relaxed on
    that surface towards equal edge lengths: gradient steps on
    sum (l - mean l)^2, each followed by projection back onto the surface
    (_project).  The plain mapping crushes the rim (edges 0.15-0.35 at
    R = 4, with 5-valent vertices on the rim); the relaxed mesh's edges
    span 0.20-0.32 about a mean of 0.253.  Triangles are oriented on the
    sphere (where the test is exact) before the mapping; neither the
    mapping nor the relaxation turns a triangle over."""
    Vs, F = icosphere(subdiv)
    Vs = Vs @ _pole_rotation(Vs[5]).T
    F = orient_outward(Vs, F)
    theta = np.arccos(np.clip(Vs[:, 2], -1.0, 1.0))
    V = evans_fung(Vs, R)
    E = edges_of(F)
    n = len(V)
    for _ in range(relax_iters):
        d = V[E[:, 0]] - V[E[:, 1]]
        ln = np.sqrt((d * d).sum(axis=1))
        g = ((ln - ln.mean()) / ln)[:, None] * d
        G = np.stack([np.bincount(E[:, 0], g[:, k], n) - np.bincount(E[:, 1], g[:, k], n) for k in range(3)],
                     axis=1)
        V, theta = _project(V - step * G, theta, R)
    return V, E, F


# The WLC spring of the reference's membrane model (Src/memfuncs.cpp:233-258)
# has a fixed persistence constant elap = 0.0005 (maincode.cpp:347), chosen
# for its shipped 600-vertex mesh, whose mean edge is 0.983753.  Its spring
# force does not shrink with the edge, so on a finer mesh the tension per
# unit length grows as 1 / (mean edge), and below an edge of about 0.35 the
# POW coefficient kappap (maincode.cpp:349-360) turns negative: the edge
# loses its repulsive core.  Coarse-graining the WLC-POW model (Fedosov,
# Caswell and Karniadakis, Biophys. J. 98 (2010) 2215) keeps the membrane's
# shear modulus by scaling the persistence length with the mesh, i.e.
# elap x mean edge held at the shipped mesh's value.
REF_ELAP, REF_MEAN_EDGE = 0.0005, 0.983753


def mean_edge(V, E):
    """mean edge length as main() prints it (maincode.cpp:239-257)"""
    V, E = np.asarray(V, float), np.asarray(E)
    return float(np.sqrt(((V[E[:, 0]] - V[E[:, 1]]) ** 2).sum(axis=1)).sum() / len(E))


def scaled_elap(V, E):
    """elap for a mesh: the reference's elap x (its mean edge / this mesh's)"""
    return REF_ELAP * REF_MEAN_EDGE / mean_edge(V, E)


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
