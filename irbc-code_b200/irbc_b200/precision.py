"""FP32-bulk against FP64: the per-observable precision study.

For each of K seeds an FP64 run and an FP32-bulk run (the same seed, so
the same random numbers) start from one shared state and advance for the
same number of steps.  The solvent of the start state carries the developed
Couette profile u_x(z) = wallspeed * z / Lz on top of its thermal
velocities, so the profile is at full strength from the first step.  Every
`every` steps each run reports the study's observables: the velocity
profile (mean solvent vx per z-layer), the solvent temperature, the
membrane area and volume, the bond count and the membrane's centre of mass.

MPCD is chaotic: after a few hundred steps an FP32 trajectory is no longer
the FP64 one but another sample of the same statistics.  So each
observable is compared as an ensemble mean over the K seeds, FP32 against
FP64, and reported with the sampling noise of that difference (the standard
error from the spread of the per-seed values, `noise_*`).  A systematic
FP32 error would stand out above the noise; an error at or below it is all
that the window can resolve.

Per run, the summaries are:
- profile: the time-averaged profile without the two wall layers;
- shear: its least-squares slope;
- temperature, area, volume, bonds: time means;
- com_velocity: least-squares slope of the centre-of-mass x over time.
`compare` reports
- profile_l2_rel = || <u32> - <u64> ||_2 / || <u64> ||_2,
- shear_rel, temperature_rel, area_rel, volume_rel: relative differences,
- bonds_abs: difference in bonds,
- com_velocity_abs: difference as a fraction of the wall speed.
"""
import ctypes as C

import numpy as np

from . import FP32, Simulation, State


def _copy_params(params, **over):
    q = type(params)()
    C.memmove(C.byref(q), C.byref(params), C.sizeof(params))
    for k, v in over.items():
        setattr(q, k, v)
    return q


def developed_couette(st, wallspeed, Lz):
    """The state with u_x(z) = wallspeed * z / Lz added to every solvent
    particle's velocity (the linear profile between the resting bottom wall
    and the top wall moving at wallspeed)."""
    out = State.from_other(st)
    out.a["svx"] = out.a["svx"] + wallspeed * out.a["sz"] / Lz
    return out


def _run(params, V, E, T, nknobs, start, steps, every, dt_step):
    sim = Simulation(params)
    sim.init(V, E, T, nknobs)      # the same mesh as the start state's
    sim.set_state(start)
    nbins = int(round(params.Lz / params.a))
    rows = []
    t = 0
    while t < steps:
        n = min(every, steps - t)
        sim.step(n)
        t += n
        ob = sim.observables()
        rows.append((t, ob[0], ob[1], ob[4], ob[5], ob[6], sim.velocity_profile(nbins)))
    sim.close()
    prof = np.mean([r[6] for r in rows], axis=0)[1:-1]
    tt = np.array([r[0] for r in rows], float) * dt_step
    cx = np.array([r[2] for r in rows], float)
    return {
        "profile": prof,
        "shear": float(np.polyfit(np.arange(prof.size, dtype=float), prof, 1)[0]),
        "temperature": float(np.mean([r[1] for r in rows])),
        "area": float(np.mean([r[3] for r in rows])),
        "volume": float(np.mean([r[4] for r in rows])),
        "bonds": float(np.mean([r[5] for r in rows])),
        "com_velocity": float(np.polyfit(tt, cx, 1)[0]) if len(tt) > 1 else 0.0,
    }


def run_study(params, V, E, T, nknobs, steps, every, seeds):
    """params: an irbc_params with precision FP64; seeds: the K seeds.
    Returns {"fp64": [summary per seed], "fp32": [...], "wallspeed": ...}."""
    first = Simulation(params)
    first.init(V, E, T, nknobs)
    start = developed_couette(first.get_state(), params.warm_speed, params.Lz)
    first.close()
    out = {"fp64": [], "fp32": [], "wallspeed": params.warm_speed}
    for seed in seeds:
        for key, over in (("fp64", {}), ("fp32", dict(precision=FP32))):
            q = _copy_params(params, seed=seed, **over)
            out[key].append(_run(q, V, E, T, nknobs, start, steps, every, params.dtmd))
    return out


def compare(study):
    """Ensemble-mean differences FP32 - FP64 and their sampling noise."""
    a, b = study["fp64"], study["fp32"]
    K = len(a)

    def stat(key):
        x = np.array([r[key] for r in a], float)
        y = np.array([r[key] for r in b], float)
        d = y.mean(axis=0) - x.mean(axis=0)
        se = np.sqrt((x.var(axis=0, ddof=1) + y.var(axis=0, ddof=1)) / K) if K > 1 else np.zeros_like(d)
        return x.mean(axis=0), d, se

    err = {}
    m, d, se = stat("profile")
    nrm = max(float(np.linalg.norm(m)), 1e-300)
    err["profile_l2_rel"] = float(np.linalg.norm(d)) / nrm
    err["noise_profile_l2_rel"] = float(np.linalg.norm(se)) / nrm
    for key in ("shear", "temperature", "area", "volume"):
        m, d, se = stat(key)
        err[key + "_rel"] = float(abs(d) / abs(m))
        err["noise_" + key + "_rel"] = float(se / abs(m))
    m, d, se = stat("bonds")
    err["bonds_abs"], err["noise_bonds_abs"] = float(abs(d)), float(se)
    m, d, se = stat("com_velocity")
    w = study["wallspeed"]
    err["com_velocity_abs"], err["noise_com_velocity_abs"] = float(abs(d) / w), float(se / w)
    err["seeds"] = K
    return err
