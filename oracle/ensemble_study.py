#!/usr/bin/env python3
"""oracle/ensemble_study.py -- TEST INFRASTRUCTURE: ensemble statistics of
the reference's configuration, from the reference itself and from the GPU
library, with the same observables computed the same way from full states.

The configuration is the reference's define.h as shipped (60 x 40 x 40 box,
960,000 solvent particles, SRD angle 135 deg, dtcd 0.02, dtmd 0.002), the
shipped 600-vertex mesh with 500 knobs, kon 0.005, koff 0.015, for `steps`
steps of main()'s loop (maincode.cpp:461-764; all inside its 250,000-step
warm-up at wall speed 0.1).  The reference runs as compiled from its own
sources with its own Mersenne Twister seeded from the clock
(oracle/_ref/cfg1_timing, -O3 -fopenmp), so each run is an independent
sample; the GPU runs the FP64 library with seeds 1..K.

Observables, sampled every `every` steps from step `start` on and averaged
over each run's window (one value per run):
  temperature  sum m |v - u_layer|^2 / (3 Ns): solvent kT from peculiar
               velocities (u_layer: the mean velocity of the particle's
               z-layer of height a)
  profile      mean solvent vx per z-layer (Lz layers): the Couette profile
  bonds        knob-ligand bonds
  rolling      the membrane's centre-of-mass x velocity, from consecutive
               samples of the unwrapped centre of mass
  area, volume Sarea, Volume

    python oracle/ensemble_study.py reference --runs 4 --out tests/golden/ensemble/reference_cfg1.json
    python oracle/ensemble_study.py gpu --runs 4
"""
import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "irbc-code_b200"))

STEPS, START, EVERY = 20000, 10000, 500


def sample(st, Lx, Ly, Lz, a=1.0, mass=1.0):
    """the observables of one full state (arrays in the reference's layout)"""
    vx, vy, vz, z = st.a["svx"], st.a["svy"], st.a["svz"], st.a["sz"]
    nl = int(Lz / a)
    layer = np.clip(np.floor(z / a).astype(np.int64), 0, nl - 1)
    cnt = np.bincount(layer, minlength=nl).astype(float)
    su = [np.bincount(layer, weights=v, minlength=nl) for v in (vx, vy, vz)]
    e = mass * float((vx * vx + vy * vy + vz * vz).sum())
    flow = sum(mass * float((s[cnt > 0] ** 2 / cnt[cnt > 0]).sum()) for s in su)
    prof = np.where(cnt > 0, su[0] / np.maximum(cnt, 1), 0.0)
    com = np.array([(st.a["x"] + st.a["ix"] * Lx).mean(), (st.a["y"] + st.a["iy"] * Ly).mean(), st.a["z"].mean()])
    return dict(temperature=(e - flow) / (3.0 * len(vx)), profile=prof, bonds=int(st.a["bondi"].sum()), com=com,
                area=float(st.s["Sarea"]), volume=float(st.s["Volume"]))


def window(samples, every, dtmd):
    """one run's window averages"""
    t = np.array([s["temperature"] for s in samples])
    prof = np.mean([s["profile"] for s in samples], axis=0)
    com = np.array([s["com"][0] for s in samples])
    roll = np.diff(com) / (every * dtmd)
    return dict(temperature=float(t.mean()), profile=[float(x) for x in prof],
                bonds=float(np.mean([s["bonds"] for s in samples])), rolling=float(roll.mean()),
                area=float(np.mean([s["area"] for s in samples])),
                volume=float(np.mean([s["volume"] for s in samples])), samples=len(samples))


def run_reference(runs, steps, start, every, threads):
    import oracle as O
    out = []
    for r in range(runs):
        R = O.Reference("cfg1_timing", threads=threads)
        p = R.p
        vf, ef, tf = O.troph_files()
        samples = []

        def cb(s):
            if start <= s <= steps and (s - start) % every == 0:
                samples.append(sample(R.get_state(s), p.Lx, p.Ly, p.Lz))
        t0 = time.time()
        wd = tempfile.mkdtemp(prefix="irbc_ens_")
        R.run(vf, ef, tf, 500, steps + 1, seed=0, on_step=cb, fast_init=1, workdir=wd)
        w = window(samples, every, p.dtmd)
        w["seconds"] = round(time.time() - t0, 1)
        out.append(w)
        print(json.dumps({"run": r, "temperature": w["temperature"], "bonds": w["bonds"],
                          "rolling": w["rolling"], "seconds": w["seconds"]}), flush=True)
        time.sleep(1.5)  # the next run's clock seed differs
    return out


def run_gpu(runs, steps, start, every, seed0=1):
    import irbc_b200 as G
    from irbc_b200 import mesh
    V, E, T = mesh.read_reference_files(*[os.path.join(ROOT, "tests", "golden", "troph600", n)
                                          for n in ("TrophV600.dat", "TrophE600.dat", "TrophT600.dat")])
    out = []
    for r in range(runs):
        p = G.default_params(seed=seed0 + r)
        sim = G.Simulation(p)
        sim.init(V, E, T, 500)
        samples = []
        # the reference is sampled at step s's TotalVA call, whose solvent
        # and vertex positions are final for step s: here after s + 1 steps
        sim.step(start + 1)
        for s in range(start, steps + 1, every):
            samples.append(sample(sim.get_state(llist=False), p.Lx, p.Ly, p.Lz))
            if s + every <= steps:
                sim.step(every)
        out.append(window(samples, every, p.dtmd))
        sim.close()
    return out


def summary(runs):
    """ensemble mean and standard error of each scalar, and of the profile"""
    out = {}
    for k in ("temperature", "bonds", "rolling", "area", "volume"):
        x = np.array([r[k] for r in runs])
        out[k] = dict(mean=float(x.mean()), se=float(x.std(ddof=1) / np.sqrt(len(x))) if len(x) > 1 else 0.0)
    P = np.array([r["profile"] for r in runs])
    out["profile"] = dict(mean=[float(x) for x in P.mean(axis=0)],
                          se=[float(x) for x in (P.std(axis=0, ddof=1) / np.sqrt(len(P)) if len(P) > 1
                                                 else np.zeros(P.shape[1]))])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("side", choices=["reference", "gpu"])
    ap.add_argument("--runs", type=int, default=4)
    ap.add_argument("--steps", type=int, default=STEPS)
    ap.add_argument("--start", type=int, default=START)
    ap.add_argument("--every", type=int, default=EVERY)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.side == "reference":
        runs = run_reference(a.runs, a.steps, a.start, a.every, a.threads)
    else:
        runs = run_gpu(a.runs, a.steps, a.start, a.every)
    res = dict(side=a.side, steps=a.steps, start=a.start, every=a.every, runs=runs, summary=summary(runs))
    if a.side == "reference":
        res["threads"] = a.threads
    text = json.dumps(res)
    if a.out:
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        with open(a.out, "w") as f:
            f.write(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
