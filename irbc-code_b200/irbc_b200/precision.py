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
- temperature_drift, area_drift, volume_drift: least-squares slope of the
  series over the run, relative to its mean, per 10,000 steps;
- bonds_series: the bond count at every sample;
- com_velocity: least-squares slope of the centre-of-mass x over time;
- rolling_mean, rolling_var: mean and variance of the centre-of-mass x
  velocity between consecutive samples.
`compare` reports
- profile_l2_rel = || <u32> - <u64> ||_2 / || <u64> ||_2,
- shear_rel, temperature_rel, area_rel, volume_rel: relative differences,
- temperature_drift_abs, area_drift_abs, volume_drift_abs: differences of
  the relative drifts per 10,000 steps,
- bonds_abs: difference in bonds; bonds_series_max_abs: the largest
  difference of the ensemble-mean bond-count series,
- com_velocity_abs, rolling_mean_abs: differences as a fraction of the
  wall speed; rolling_var_rel: relative difference of the variances.
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
    steps_at = np.array([r[0] for r in rows], float)
    tt = steps_at * dt_step
    cx = np.array([r[2] for r in rows], float)

    def drift(col):
        y = np.array([r[col] for r in rows], float)
        return float(np.polyfit(steps_at, y, 1)[0] * 1e4 / np.mean(y)) if len(y) > 1 else 0.0
    vel = np.diff(cx) / np.diff(tt) if len(tt) > 1 else np.zeros(1)
    return {
        "profile": prof,
        "shear": float(np.polyfit(np.arange(prof.size, dtype=float), prof, 1)[0]),
        "temperature": float(np.mean([r[1] for r in rows])),
        "area": float(np.mean([r[3] for r in rows])),
        "volume": float(np.mean([r[4] for r in rows])),
        "bonds": float(np.mean([r[5] for r in rows])),
        "temperature_drift": drift(1),
        "area_drift": drift(3),
        "volume_drift": drift(4),
        "bonds_series": np.array([r[5] for r in rows], float),
        "com_velocity": float(np.polyfit(tt, cx, 1)[0]) if len(tt) > 1 else 0.0,
        "rolling_mean": float(np.mean(vel)),
        "rolling_var": float(np.var(vel)),
    }


def run_study(params, V, E, T, nknobs, steps, every, seeds):
    """params: an irbc_params with precision FP64; seeds: the K seeds.
    The wall moves at warm_speed for the first warm_steps steps and at walls
    after (maincode.cpp:463-470).  Returns {"fp64": [summary per seed],
    "fp32": [...], "wallspeed": ...}."""
    ws = params.warm_speed if params.warm_steps > 0 else params.walls
    first = Simulation(params)
    first.init(V, E, T, nknobs)
    start = developed_couette(first.get_state(), ws, params.Lz)
    first.close()
    out = {"fp64": [], "fp32": [], "wallspeed": ws}
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
    for key in ("temperature_drift", "area_drift", "volume_drift"):
        m, d, se = stat(key)
        err[key + "_abs"], err["noise_" + key + "_abs"] = float(abs(d)), float(se)
    m, d, se = stat("bonds")
    err["bonds_abs"], err["noise_bonds_abs"] = float(abs(d)), float(se)
    m, d, se = stat("bonds_series")
    err["bonds_series_max_abs"], err["noise_bonds_series_max_abs"] = float(np.max(np.abs(d))), float(np.max(se))
    w = study["wallspeed"]
    for key in ("com_velocity", "rolling_mean"):
        m, d, se = stat(key)
        err[key + "_abs"], err["noise_" + key + "_abs"] = float(abs(d) / w), float(se / w)
    m, d, se = stat("rolling_var")
    err["rolling_var_rel"] = float(abs(d) / max(abs(m), 1e-300))
    err["noise_rolling_var_rel"] = float(se / max(abs(m), 1e-300))
    err["seeds"] = K
    return err


def main(argv=None):
    """python -m irbc_b200.precision --config large --seeds 16 --steps 10000 --every 500

    config "reference": the reference's define.h configuration (960,000
    particles, the shipped 600-vertex mesh, 500 knobs), wall at the
    warm-up speed 0.1; config "large": the large single simulation
    (irbc_b200.workloads.LARGE) with its shear walls/Lz = 0.01 from the
    first step.  Prints one JSON line: the comparison and the settings."""
    import argparse
    import json
    import os
    import time
    from . import default_params, mesh, workloads
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["reference", "large"], default="large")
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--every", type=int, default=500)
    a = ap.parse_args(argv)
    if a.config == "large":
        p = workloads.large_params(seed=1, precision=0, warm_steps=0)
        V, E, T = workloads.large_mesh()
        nknobs = workloads.LARGE["nknobs"]
    else:
        p = default_params(onrate=0.005, offrate=0.015, Nt=600)
        here = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        V, E, T = mesh.read_reference_files(*[os.path.join(here, "tests", "golden", "troph600", n)
                                              for n in ("TrophV600.dat", "TrophE600.dat", "TrophT600.dat")])
        nknobs = 500
    t0 = time.time()
    study = run_study(p, V, E, T, nknobs, a.steps, a.every, seeds=tuple(range(101, 101 + a.seeds)))
    err = compare(study)
    print(json.dumps(dict(config=a.config, seeds=a.seeds, steps=a.steps, every=a.every,
                          wallspeed=study["wallspeed"], seconds=round(time.time() - t0, 1), compare=err)))


if __name__ == "__main__":
    main()
