"""The workloads of the benchmark and of the tests that check it at size.

LARGE is the large single simulation: a 128 x 64 x 64 box at 10 solvent
particles per cell (5,242,880), SRD angle 130 deg, dtcd 0.025 (12 streaming
steps per collision), dtmd 0.002, moving wall 0.64 (shear walls/Lz = 0.01),
and one 2562-vertex Evans-Fung discocyte of radius 4 (mesh.discocyte) with
1000 knobs, kon 0.005, koff 0.015.  Every other parameter is define.h's
(irbc_params_default), except the WLC persistence constant elap, which is
scaled to the mesh (mesh.scaled_elap: 0.00194 against the 0.0005 the
reference hard-codes for its 0.98-edge mesh).  With the literal 0.0005 the
discocyte's 0.25-long edges have negative POW coefficients and the cell
blows up after a few hundred to about 1,400 steps in the reference's own
arithmetic; with the scaled value it runs for 50,000 steps.
"""
import math

LARGE = dict(Lx=128.0, Ly=64.0, Lz=64.0, Ns=5242880, alpha_deg=130.0, dtcd=0.025, dtmd=0.002, walls=0.64,
             nknobs=1000, kon=0.005, koff=0.015, R=4.0)


def large_mesh():
    """(V, E, T) of the discocyte"""
    from . import mesh
    return mesh.discocyte(4, LARGE["R"])


def large_params(seed, precision=0, **over):
    """irbc_params of the large simulation (over: fields to replace)"""
    from . import default_params, mesh
    W = LARGE
    V, E, _ = large_mesh()
    a = math.radians(W["alpha_deg"])
    kw = dict(Lx=W["Lx"], Ly=W["Ly"], Lz=W["Lz"], Ns=W["Ns"], cosalpha=math.cos(a), sinalpha=math.sin(a),
              dtcd=W["dtcd"], dtmd=W["dtmd"], walls=W["walls"], onrate=W["kon"], offrate=W["koff"], Nt=len(V),
              elap=mesh.scaled_elap(V, E), seed=seed, precision=precision)
    kw.update(over)
    return default_params(**kw)


def replica_params(Lx, Ly, Lz, seed, kon, koff, precision=1, walls_frac=0.01, mesh_ve=None):
    """A batched or served replica: box Lx x Ly x Lz at 10 particles per
    cell, SRD angle 130 deg, dtcd 0.025, dtmd 0.002, wall speed walls_frac x
    Lz.  mesh_ve = (V, E) of a mesh other than the shipped one: elap scaled
    to it."""
    from . import default_params, mesh
    a = math.radians(130.0)
    kw = dict(Lx=float(Lx), Ly=float(Ly), Lz=float(Lz), Ns=int(Lx * Ly * (Lz + 1) * 10), cosalpha=math.cos(a),
              sinalpha=math.sin(a), dtcd=0.025, dtmd=0.002, walls=walls_frac * Lz, onrate=kon, offrate=koff,
              seed=seed, precision=precision)
    if mesh_ve is not None:
        kw["Nt"] = len(mesh_ve[0])
        kw["elap"] = mesh.scaled_elap(*mesh_ve)
    return default_params(**kw)
