#!/usr/bin/env python3
"""oracle/ref_bench.py -- TEST INFRASTRUCTURE: times the reference's own
OpenMP step on this machine's host cores (bench.py's CPU-baseline leg and
`bench.py --impl reference`).

Runs the reference's unmodified main() (compiled in oracle/_ref/<variant>
with its own Mersenne Twister, -O3 -fopenmp) for warm-up + `steps` steps and
reports solvent particle-steps/s over the timed steps, measured between the
TotalVA calls of consecutive steps (maincode.cpp:602), so every timed step
is a whole loop iteration including its share of collisions (every csteps
steps).  Set-up is excluded; its solvent inside/outside pass runs on all
threads (same flags as the reference's serial loop).  Prints one JSON line.
"""
import argparse
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "irbc-code_b200"))


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--variant", default="large_timing")
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--nknobs", type=int, default=0, help="default: 500 on the 600-vertex mesh, 1000 otherwise")
    ap.add_argument("--onrate", type=float, default=0.005)
    ap.add_argument("--offrate", type=float, default=0.015)
    a = ap.parse_args()
    threads = a.threads or host_threads()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle as O
    from irbc_b200 import mesh
    R = O.Reference(a.variant, threads=threads)
    wd = tempfile.mkdtemp(prefix="irbc_refbench_")
    nknobs = a.nknobs or (500 if R.p.Nt == 600 else 1000)
    if nknobs > R.p.Nt:
        raise SystemExit("the reference's knob loop never ends with more knobs than vertices")
    if R.p.Nt == 600:
        vf, ef, tf = O.troph_files()
    else:
        V, E, T = mesh.discocyte()
        if len(V) != R.p.Nt:
            raise SystemExit("no mesh with %d vertices" % R.p.Nt)
        vf, ef, tf = mesh.write_reference_files(wd, V, E, T)
    t0 = time.perf_counter()
    stop = a.warmup + a.steps
    R.run(vf, ef, tf, nknobs, stop, seed=int(time.time()), onrate=a.onrate, offrate=a.offrate,
          fast_init=1, workdir=wd)
    wall = time.perf_counter() - t0
    ts = R.step_times()
    # ts[s] = time of the TotalVA call of step s; steps warmup+1 .. stop are whole iterations
    dt = ts[stop] - ts[a.warmup]
    ns = R.p.Ns
    out = dict(value=ns * a.steps / dt, unit="particle-steps/s", cores=threads, steps=a.steps,
               warmup=a.warmup, seconds=dt, Ns=ns, box=[R.p.Lx, R.p.Ly, R.p.Lz], nv=R.p.Nt,
               init_s=ts[0] - 0.0, total_wall_s=wall, variant=a.variant)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
