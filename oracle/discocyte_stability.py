#!/usr/bin/env python3
"""oracle/discocyte_stability.py -- TEST INFRASTRUCTURE: the CPU oracle
(which equals the reference bit for bit) run for many steps on the large
workload's membrane, to show whether the discocyte stays physical.

The setting is the reference's own step with the large workload's
membrane: the 2562-vertex discocyte of irbc_b200.mesh.discocyte with 1000
knobs, SRD angle 130 deg, dtcd 0.025, dtmd 0.002, walls/Lz 0.01, kon 0.005,
koff 0.015, in a 32^3 box with 40,000 solvent particles (the thin solvent
keeps the CPU run to minutes; the membrane sees the same collisions and
thermostat).  It runs once with the WLC persistence constant the reference
hard-codes (elap 0.0005, maincode.cpp:347) and once with elap scaled to the
mesh (irbc_b200.mesh.scaled_elap), printing one JSON line every `every`
steps (area, volume, largest vertex speed, shortest and longest edge,
bonds) until the state goes non-finite or `steps` steps have run.

    python oracle/discocyte_stability.py --steps 50000 --every 1000
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "irbc-code_b200"))


def run(elap, steps, every, seed=31, box=32.0, ns=40000):
    import oracle as O
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte()
    a = math.radians(130.0)
    op = O.default_params(Lx=box, Ly=box, Lz=box, Ns=ns, Nt=len(V), dtcd=0.025, walls=0.01 * box,
                          cosalpha=math.cos(a), sinalpha=math.sin(a), onrate=0.005, offrate=0.015, elap=elap)
    orc = O.Oracle(op, seed)
    orc.init(V, E, T, 1000)
    t0 = time.time()
    done = 0
    while done < steps:
        k = min(every, steps - done)
        orc.step(k)
        done += k
        st = orc.get_state()
        v = np.sqrt(st.a["vx"] ** 2 + st.a["vy"] ** 2 + st.a["vz"] ** 2)
        P = np.stack([st.a["x"] + st.a["ix"] * box, st.a["y"] + st.a["iy"] * box, st.a["z"]], axis=1)
        ln = np.linalg.norm(P[E[:, 0]] - P[E[:, 1]], axis=1)
        row = dict(elap=elap, step=done, seconds=round(time.time() - t0, 1), area=st.s["Sarea"],
                   volume=st.s["Volume"], vmax=float(v.max()), lmin=float(ln.min()), lmax=float(ln.max()),
                   bonds=int(st.a["bondi"].sum()), finite=bool(np.isfinite(v).all()))
        print(json.dumps(row), flush=True)
        if not row["finite"]:
            break


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--only", choices=["literal", "scaled"], default=None)
    a = ap.parse_args()
    from irbc_b200 import mesh
    V, E, _ = mesh.discocyte()
    for name, elap in (("literal", mesh.REF_ELAP), ("scaled", mesh.scaled_elap(V, E))):
        if a.only in (None, name):
            run(elap, a.steps, a.every)


if __name__ == "__main__":
    main()
