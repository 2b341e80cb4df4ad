"""Mesh tooling (no GPU): the discocyte generator's topology and
orientation, the reference file format round trip, and the shipped
trophozoite mesh's conventions that the generator follows."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "irbc-code_b200"))

import helpers as H  # noqa: E402


def _closed_manifold(E, T, nv):
    # every edge in exactly two triangles, every directed edge once
    und = {}
    directed = set()
    for a, b, c in T:
        for u, v in ((a, b), (b, c), (c, a)):
            assert (u, v) not in directed
            directed.add((u, v))
            key = (min(u, v), max(u, v))
            und[key] = und.get(key, 0) + 1
    assert all(n == 2 for n in und.values())
    assert set(und) == {(int(a), int(b)) for a, b in E}
    assert nv - len(E) + len(T) == 2  # Euler characteristic of a sphere


def _outward(V, T):
    c = V.mean(axis=0)
    A, B, C = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    n = np.cross(B - A, C - A)
    return ((((A + B + C) / 3.0) - c) * n).sum(axis=1)


def test_discocyte_topology_and_orientation():
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte()
    assert (len(V), len(E), len(T)) == (2562, 7680, 5120)
    assert (E[:, 0] < E[:, 1]).all()
    _closed_manifold(E, T, len(V))
    # every triangle outward, so they enclose a positive volume
    assert (_outward(V, T) > 0).all()
    A, B, C = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    vol = np.einsum("ij,ij->i", A, np.cross(B, C)).sum() / 6.0
    assert vol > 0
    # on the Evans-Fung surface of radius 4: |z| = h(r) at every vertex
    r = np.hypot(V[:, 0], V[:, 1])
    rho2 = np.clip((r / 4.0) ** 2, 0, 1)
    h = 2.0 * np.sqrt(1 - rho2) * (mesh.EF_C0 + mesh.EF_C1 * rho2 + mesh.EF_C2 * rho2 ** 2)
    assert np.max(np.abs(np.abs(V[:, 2]) - h)) < 1e-12
    assert 3.99 < r.max() <= 4.0 + 1e-12
    assert 0.5 < V[:, 2].max() - V[:, 2].min() < 4.0


def test_discocyte_edges_are_near_uniform():
    """The relaxed mesh: edges within about +-25% of their mean (the plain
    mapping of the icosphere spans 0.15-0.35), and none of the twelve
    5-valent vertices on the rim."""
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte()
    ln = np.linalg.norm(V[E[:, 0]] - V[E[:, 1]], axis=1)
    assert ln.min() > 0.75 * ln.mean() and ln.max() < 1.3 * ln.mean()
    assert ln.std() < 0.1 * ln.mean()
    valence = np.bincount(E.ravel())
    assert (valence == 5).sum() == 12
    assert np.hypot(V[valence == 5, 0], V[valence == 5, 1]).max() < 0.9 * 4.0
    # the persistence constant scaled to the mesh keeps the shipped mesh's
    # elap x mean edge
    assert abs(mesh.scaled_elap(V, E) * mesh.mean_edge(V, E) - 0.0005 * 0.983753) < 1e-15


def test_reference_file_round_trip(tmp_path):
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte(subdiv=2)
    pv, pe, pt = mesh.write_reference_files(str(tmp_path), V, E, T)
    V2, E2, T2 = mesh.read_reference_files(pv, pe, pt)
    assert np.array_equal(E2, E) and np.array_equal(T2, T)
    assert np.max(np.abs(V2 - V)) < 1e-9
    Va, _, _ = mesh.discocyte_as_read(subdiv=2)
    assert np.array_equal(Va, V2)


def test_shipped_mesh_follows_the_same_conventions():
    V, E, T = H.troph()
    V, E, T = np.asarray(V), np.asarray(E), np.asarray(T)
    assert (len(V), len(E), len(T)) == (600, 1794, 1196)
    assert (E[:, 0] < E[:, 1]).all()
    _closed_manifold(E, T, len(V))
    assert (_outward(V, T) > 0).mean() > 0.95
