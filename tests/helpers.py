"""Shared test helpers: build matching oracle / GPU simulations."""
import numpy as np

import oracle as O


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def to_irbc_params(op, seed, precision=0):
    import irbc_b200 as G
    p = G.default_params()
    for name, _ in O.Params._fields_:
        if name != "pad_":
            setattr(p, name, getattr(op, name))
    p.seed = seed
    p.precision = precision
    return p


def troph():
    return O.load_mesh_files(*O.troph_files())


def make_oracle(ns=40000, seed=11, onrate=0.005, offrate=0.015, nknobs=500, **over):
    op = O.default_params(Ns=ns, onrate=onrate, offrate=offrate, **over)
    orc = O.Oracle(op, seed)
    V, E, T = troph()
    orc.init(V, E, T, nknobs)
    return op, orc


def gpu_like(op, orc, seed, precision=0, state=None):
    """GPU simulation with the oracle's parameters, mesh and state."""
    import irbc_b200 as G
    sim = G.Simulation(to_irbc_params(op, seed, precision))
    sim.set_mesh(orc.get_mesh())
    st = state if state is not None else orc.get_state()
    sim.set_state(G.State.from_other(st))
    return sim


def oracle_params(p):
    """oracle Params with the fields of the irbc_params p"""
    op = O.default_params()
    for name, _ in O.Params._fields_:
        if name != "pad_":
            setattr(op, name, getattr(p, name))
    return op


def oracle_like(sim, p):
    """an oracle with the GPU simulation's parameters, mesh and state"""
    op = oracle_params(p)
    orc = O.Oracle(op, p.seed)
    a, sc = sim.get_mesh_arrays()
    M = O.MeshArrays(sim.nv, len(a["e1"]), len(a["t1"]))
    for k in M.a:
        M.a[k][:] = a[k]
    M.s.update(sc)
    orc.set_mesh(M)
    orc.set_state(oracle_state(sim.get_state()))
    return op, orc


def oracle_state(st):
    """an oracle State holding the arrays and scalars of a GPU state"""
    ost = O.State(st.ns, st.nv, st.nlig, st.ncell, max(1, st.a["lidx"].size))
    for k, v in st.a.items():
        ost.a[k] = np.ascontiguousarray(v).copy()
    for k, v in st.s.items():
        ost.s[k] = np.array(v).copy() if isinstance(v, np.ndarray) else v
    return ost


def rel_err(a, b):
    """normwise relative error max|a-b| / max|b|"""
    a, b = np.asarray(a), np.asarray(b)
    if a.size == 0:
        return 0.0
    d = np.max(np.abs(a - b))
    s = np.max(np.abs(b))
    return float(d / s) if s > 0 else float(d)


FLOAT_FIELDS = ("sx", "sy", "sz", "svx", "svy", "svz", "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz",
                "poff", "pon")
INT_FIELDS = ("spid", "sindio", "pid", "ix", "iy", "bondi", "bondl", "knob", "ligi", "llen")


def compare(gpu, ref, rtol=1e-12, fields=None, skip=()):
    """Returns a dict of failures: float fields normwise-relative above rtol,
    integer fields with any mismatch, llist entries."""
    bad = {}
    for k in fields or (FLOAT_FIELDS + INT_FIELDS):
        if k in skip or k not in gpu.a or k not in ref.a:
            continue
        a, b = gpu.a[k], ref.a[k]
        if a.shape != b.shape:
            bad[k] = ("shape", a.shape, b.shape)
        elif a.dtype.kind == "f":
            e = rel_err(a, b)
            if not (e <= rtol):
                bad[k] = e
        else:
            n = int((a != b).sum())
            if n:
                bad[k] = n
    if "lidx" in gpu.a and "lidx" in ref.a and "llen" not in skip:
        la = gpu.a["lidx"][: int(gpu.a["llen"].sum())]
        lb = ref.a["lidx"][: int(ref.a["llen"].sum())]
        if la.shape != lb.shape or (la != lb).any():
            bad["lidx"] = "differs"
    for k in ("para", "paraV", "paraft", "parafdt"):
        e = rel_err(gpu.s[k], ref.s[k])
        if not (e <= rtol):
            bad[k] = e
    for k in ("Sarea", "Volume"):
        if abs(gpu.s[k] - ref.s[k]) > rtol * abs(ref.s[k]):
            bad[k] = (gpu.s[k], ref.s[k])
    for k in ("paradx", "parady", "paraid"):
        if gpu.s[k] != ref.s[k]:
            bad[k] = (gpu.s[k], ref.s[k])
    return bad
