#!/usr/bin/env python3
"""bench.py -- solvent particle-steps/s of the iRBC timestep on B200.

Workload (the reference's large single-simulation configuration): box
128 x 64 x 64 cells, 10 solvent particles per cell (5,242,880), SRD angle
130 deg, dtcd 0.025 (12 streaming steps per collision), dtmd 0.002, moving
wall 0.64 (shear 0.01), one 2562-vertex Evans-Fung discocyte of radius 4
with 1000 knobs, kon 0.005, koff 0.015.  Synthetic data: positions and
velocities from the seeded draw stream, the discocyte from
irbc_b200/mesh.py.

A "step" is one reference timestep (maincode.cpp:461-764): streaming with
bounce-back of every particle, the membrane update, every 12th step the
collision and every 390th the triangle-list update (llistupdate).  The
default 780 timed steps hold 65 collisions and 2 list updates, so every
part of the step enters at its own frequency.  `value` = Ns * steps * ranks / max-over-ranks device time of the
timed steps (CUDA events on the library's stream).  The solvent state
(~630 MB in FP64) is larger than L2 (126 MB), so no flush is needed between
steps.  N > 1 GPUs run independent replicas (different seeds), no
collective in the data path.

`--impl reference` times the reference's own OpenMP code (oracle/_ref, the
same box, Ns, mesh, angle and dt compiled into its define.h) on the host
cores.

Two more objects ride on the same JSON line (skip with --no-batch /
--no-serve): "batched", 64 replicas of uneven box (Lx 32..96, Ly = Lz = 32,
the shipped 600-vertex mesh, seeded knob counts and rates, FP32 bulk)
stepped together through irbc_batch against the same replicas stepped one
at a time; and "served", Poisson-arriving sweep requests admitted by the
request server by device-memory footprint, with p50/p99 completion
latency, sims/hr and the aggregate rate against running each request
alone.  Both use shortened step counts so that the run stays within
minutes; the requests' shapes, sizes and parameter ranges are the
workload's.
"""
import argparse
import json
import os
# many replicas' streams need more than the default 8 hardware queues;
# read by CUDA when the process first uses it
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
# every kernel loaded when the context is created, so that no first use
# (a list update, a re-sort) loads one inside the timed steps
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "irbc-code_b200"))

METRIC = "MPCD solvent particle-steps/s (large single simulation, 128x64x64, 5.24M particles)"
UNIT = "particle-steps/s"


def workload_config():
    from irbc_b200 import mesh, workloads
    W = workloads.LARGE
    V, E, _ = workloads.large_mesh()
    return dict(workload="large single simulation: box 128x64x64, 5242880 solvent, 2562-vertex discocyte "
                         "R=4, 1000 knobs, alpha 130 deg, dtcd 0.025, dtmd 0.002, walls 0.64",
                Lx=W["Lx"], Ly=W["Ly"], Lz=W["Lz"], Ns=W["Ns"], alpha_deg=W["alpha_deg"], dtcd=W["dtcd"],
                dtmd=W["dtmd"], walls=W["walls"], nknobs=W["nknobs"], kon=W["kon"], koff=W["koff"],
                elap=round(mesh.scaled_elap(V, E), 8), mesh="icosphere level 4 relaxed on the Evans-Fung surface")


# whole collision cycles: a collision every 12 steps (dtcd / dtmd)
CYCLE = 12


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.start = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            # nvidia-smi's start-up (NVML initialisation) stalls the
            # driver: wait for its first sample before the timed region
            # begins, and keep only the samples taken inside it
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.start = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, mem, reasons = [], 0.0, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        inside = self.lines[self.start:] or self.lines
        for l in inside:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
                if len(f) > 9:
                    mem.append(float(f[9]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm.sort()
        mem.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "mem_mhz": mem[len(mem) // 2] if mem else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_warm(device, seconds):
    """Device-to-device copies of a 1 GiB buffer for about `seconds`."""
    try:
        import torch
        a = torch.empty(1 << 28, dtype=torch.float32, device="cuda:%d" % device)
        b = torch.empty_like(a)
        t0 = time.time()
        while time.time() - t0 < seconds:
            for _ in range(8):
                b.copy_(a)
            torch.cuda.synchronize(device)
        del a, b
        torch.cuda.empty_cache()
    except Exception:
        pass


def make_params(G, seed, precision):
    from irbc_b200 import workloads
    return workloads.large_params(seed, precision)


def dist_setup():
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL
    when CUDA is there, gloo otherwise (the CPU tests of the N > 1 path).
    Ranks run independent replicas: the process group only times them."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def replica_seed(rank):
    """each rank's replica draws from its own seed"""
    return 1234 + 7919 * rank


def aggregate(ns, steps, world, t_ms):
    """whole-job particle-steps/s: every rank's particles over the slowest rank's time"""
    return ns * steps * world / (t_ms * 1e-3)


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(steps=12, warmup=1, variant="large_timing"):
    """The reference's OpenMP code on this host's cores, bounded sample."""
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "ref_bench.py"), "--variant", variant,
           "--steps", str(steps), "--warmup", str(warmup)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1500)
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        d = json.loads(line)
        return d
    except Exception as e:  # reported, never silently replaced
        return {"error": "%s: %s" % (type(e).__name__, str(e)[:200])}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    # whole collision cycles (a collision every 12 steps): 12, or 24 when
    # the run asks for at least 24 steps
    steps = 24 if args.steps >= 24 else 12
    warm = min(args.warmup, 1)
    d = cpu_baseline(steps, warm)
    if "error" in d:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU run failed: " + d["error"]}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * d["seconds"] / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(), parallelism="host OpenMP, %d threads" % d["cores"]),
        "cpu_baseline": {"value": d["value"], "unit": UNIT, "cores": d["cores"], "kind": "reference",
                         "sample": "%d whole timesteps after %d warm-up of the reference's main loop "
                                   "(oracle/_ref/large_timing, -O3 -fopenmp, its own Mersenne Twister); "
                                   "set-up excluded" % (steps, warm)},
        "e2e": {"value": d["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    world, rank, local = dist_setup()
    import numpy as np
    import irbc_b200 as G
    from irbc_b200 import workloads
    precision = G.FP32 if args.precision == "fp32" else G.FP64
    # whole collision cycles, so that the timed steps hold the collision at
    # its own frequency
    steps = -(-args.steps // CYCLE) * CYCLE
    p = make_params(G, seed=replica_seed(rank), precision=precision)
    p.device = local
    sim = G.Simulation(p)
    V, E, T = workloads.large_mesh()
    sim.init(V, E, T, workloads.LARGE["nknobs"])
    sim.step(args.warmup)
    sim.sync()
    # the end-to-end leg below replays the same steps from this state
    start = sim.get_state() if args.e2e else None
    # keep the GPU busy for a second before the timed steps (memory and SM
    # clocks leave their idle states), without advancing the simulation
    gpu_warm(local, 1.0)
    launches0 = int(sim.L.irbc_launch_count(sim.h))
    # the timed steps: two CUDA events on the simulation's stream, bracketed
    # by a synchronize and a barrier over the ranks on both sides (the
    # per-phase profile is taken in a separate window below)
    with ClockSampler(local) as clocks:
        sim.sync()
        barrier(world)
        sim.timer_begin()
        h0 = time.perf_counter()
        sim.step(steps)
        host_enqueue_s = time.perf_counter() - h0
        t_local = sim.timer_end()
        sim.sync()
        barrier(world)
    launches = int(sim.L.irbc_launch_count(sim.h)) - launches0
    t_ms = reduce_max(t_local, world)
    ns = workloads.LARGE["Ns"]
    value = aggregate(ns, steps, world, t_ms)
    # the state must still be physical after the timed steps
    finite = bool(np.isfinite(sim.observables()[:6]).all())
    # per-phase and per-kernel times: a short profiled window right after
    # the timed steps
    sim.profile_begin()
    sim.step(48)
    kprof = sim.profile_end()
    # roofline of the dominant kernel, the bulk streaming kernel (one launch
    # per step over every particle): its algorithmic bytes per particle are
    # the stream's state read and positions written -- FP64: positions 3 x 8
    # and velocities 3 x 8 read, positions 3 x 8 written = 72 B; FP32: two
    # float4 read, one written = 48 B (the 32-byte FP64 velocity record
    # carries the reference index too, so the kernel moves 80 B, counted
    # here as 72) -- divided by its CUDA-event time per launch
    bpp = 72 if precision == G.FP64 else 48
    bulk_avg_ms = kprof["bulk_ms"] / max(1, kprof["bulk_launches"])
    achieved = ns * bpp / (bulk_avg_ms * 1e-3) / 1e9
    # the whole step against the same bound: streaming every step plus the
    # collision's read and write once per 10-12 steps (79.2 B FP64, 52.8 B
    # FP32 per particle-step), at the measured particle-steps/s
    step_bpp = 79.2 if precision == G.FP64 else 52.8
    peak, kind = peaks()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "stream_traffic.json")
    if os.path.exists(tfile):
        try:
            tj = json.load(open(tfile))
            traffic = tj.get("fp64" if precision == G.FP64 else "fp32")
        except Exception:
            traffic = None
    # end to end through the C ABI with host buffers: the full state in from
    # page-locked memory, every step the RBCdata record out, the final state out
    e2e = None
    if args.e2e:
        e2e = run_e2e(G, sim, start, steps, workloads.LARGE["Ns"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "steps_requested": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if precision == G.FP64 else "f32", "data": "synthetic",
        "config": dict(workload_config(), parallelism="replicas x%d" % world if world > 1 else "single GPU",
                       l2="state larger than L2 (no flush needed)",
                       timed="whole collision cycles: the requested steps rounded up to a multiple of 12"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "k_stream_fast" if precision == G.FP64 else "k_stream_f",
                     "bytes_per_particle": bpp, "units_per_launch": ns, "peak_kind": kind,
                     "kernel_ms_avg": bulk_avg_ms,
                     "step_bytes_per_particle_step": step_bpp,
                     "step_achieved": value / world * step_bpp / 1e9,
                     "step_frac": value / world * step_bpp / 1e9 / peak},
        "phase_ms_per_step": {"stream": kprof["stream_ms"] / 48, "collide": kprof["collide_ms"] / 48,
                              "membrane": kprof["membrane_ms"] / 48,
                              "window": "48 steps after the timed steps"},
        "gpu_launches": launches,
        "host_enqueue_ms_per_step": 1e3 * host_enqueue_s / steps,
        "clocks": clocks.summary(),
        "state_finite": finite,
    }
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and not args.no_cpu_baseline:
        d = cpu_baseline(12, 1)
        if "error" in d:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                    "sample": "failed: " + d["error"]}
        else:
            line["cpu_baseline"] = {"value": d["value"], "unit": UNIT, "cores": d["cores"], "kind": "reference",
                                    "sample": "12 whole timesteps (one collision) of the reference's main loop on "
                                              "the same workload, after 1 warm-up step; set-up excluded"}
    sim.close()
    if world == 1 and args.batch:
        line["batched"] = run_batched(G)
    if world == 1 and args.serve:
        # the server's own default schedule (the pool): the batched leg's
        # tuned schedule suits its uniform replicas, not the served mix of
        # boxes and meshes
        line["served"] = run_served(G, scale=args.serve_scale)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


TROPH = [os.path.join(ROOT, "tests", "golden", "troph600", n) for n in ("TrophV600.dat", "TrophE600.dat",
                                                                      "TrophT600.dat")]


def run_batched(G, nrep=64, steps=240, nthreads=8):
    """64 replicas of uneven box (Lx in 32..96, Ly = Lz = 32 cells, 10 per
    cell), the 600-vertex mesh, knobs in 100..600 (the reference's knob
    placement cannot place more knobs than the mesh has vertices), kon
    log-uniform in 1e-4..1e-1, koff in 1e-3..1e-1, FP32 bulk.  Timed: every
    replica alone on the plain path, one after another (the plain value);
    the batch with one launch per phase over all replicas (the default
    schedule); the batch through the pool of host threads (fused = 0); and
    the batch under the schedule irbc_batch_autotune chose on the replicas
    themselves.  Each timed stretch is `steps` steps (whole collision
    cycles) after a warm-up, host wall clock with the device work waited
    for."""
    import numpy as np
    from irbc_b200 import mesh, workloads
    V, E, T = mesh.read_reference_files(*TROPH)
    rng = np.random.default_rng(2024)
    sims = []
    for r in range(nrep):
        Lx = int(rng.integers(32, 97))
        kon, koff = 10 ** rng.uniform(-4, -1), 10 ** rng.uniform(-3, -1)
        p = workloads.replica_params(Lx, 32, 32, 5000 + r, kon, koff, precision=G.FP32)
        s = G.Simulation(p)
        s.init(V, E, T, int(rng.integers(100, 601)))
        sims.append(s)
    ns = [s.params.Ns for s in sims]
    total = sum(ns)
    # plain path: every replica alone, one after the other
    t_alone = 0.0
    for s in sims:
        s.step(48)
        s.sync()
        t = time.perf_counter()
        s.step(steps)
        s.sync()
        t_alone += time.perf_counter() - t
    plain = total * steps / t_alone

    def timed(b, n):
        t = time.perf_counter()
        b.step(n)
        return time.perf_counter() - t

    b = G.Batch(nthreads=nthreads)
    for s in sims:
        b.add(s)
    b.step(48)  # the cohort's tables built, every kernel loaded
    l0 = sims[0].launch_count()
    dt_fused = timed(b, steps)
    launches = (sims[0].launch_count() - l0) / steps
    b.set_schedule(fused=0)
    b.step(48)
    dt_pool = timed(b, steps)
    b.set_schedule(fused=1)
    # the launch schedule tuned on the replicas themselves (its trial steps
    # advance them like any other), then the same stretch timed again
    t = time.perf_counter()
    sched, tune_steps = b.autotune(trial_steps=48, repeats=2)
    tune_s = time.perf_counter() - t
    dt = timed(b, steps)
    agg = total * steps / dt
    finite = all(bool(np.isfinite(s.observables()[:6]).all()) for s in sims)
    health = [s.health() for s in sims]
    b.close()
    for s in sims:
        s.close()
    peak, kind = peaks()
    return {"metric": "aggregate solvent particle-steps/s, %d replicas stepped together" % nrep,
            "value": agg, "unit": UNIT, "replicas": nrep, "particles": int(total), "steps": steps,
            "seconds": dt, "ms_per_batch_step": 1e3 * dt / steps,
            "plain_value": plain, "plain_sample": "all %d replicas alone, one after another" % nrep,
            "vs_plain": agg / plain,
            "fused_default_value": total * steps / dt_fused, "pool_value": total * steps / dt_pool,
            "launches_per_batch_step": launches,
            "roofline": {"bytes_per_particle_step": 52.8, "achieved_gbs": agg * 52.8 / 1e9, "peak": peak,
                         "peak_kind": kind, "frac": agg * 52.8 / 1e9 / peak},
            "host_threads": nthreads, "dtype": "f32-bulk", "state_finite": finite, "healthy": not any(health),
            "schedule": sched,
            "autotune": {"seconds": tune_s, "steps": tune_steps, "trial_steps": 48, "repeats": 2},
            "config": "Lx uniform 32..96, Ly = Lz = 32, 10/cell, 600-vertex mesh, knobs 100..600, "
                      "kon log-U 1e-4..1e-1, koff log-U 1e-3..1e-1, seeded"}


def served_requests(G, nreq, rate, scale, seed=77):
    """The serving workload's requests: Poisson arrivals (mean `rate`/s),
    kon log-uniform in 1e-4..1e-1, koff in 1e-3..1e-1, knobs 50..1000 (at
    most the mesh's vertices), shear walls/Lz in 0.002..0.02, Lx 32..128,
    Ly = Lz in 24..48 cells, the 600-vertex trophozoite or the 2562-vertex
    discocyte, FP32 bulk, and 10k..200k steps times `scale` (rounded to
    whole 24-step stretches).  Returns (params, V, E, T, knobs, steps, gap)."""
    import numpy as np
    from irbc_b200 import mesh, workloads
    meshes = [mesh.read_reference_files(*TROPH), mesh.discocyte()]
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(nreq):
        which = int(rng.integers(0, 2))
        V, E, T = meshes[which]
        Ly = int(rng.integers(24, 49))
        p = workloads.replica_params(int(rng.integers(32, 129)), Ly, Ly, 9000 + k, 10 ** rng.uniform(-4, -1),
                                     10 ** rng.uniform(-3, -1), precision=G.FP32,
                                     walls_frac=rng.uniform(0.002, 0.02), mesh_ve=(V, E) if which else None)
        nk = int(rng.integers(50, min(1000, len(V)) + 1))
        steps = max(24, int(round(rng.uniform(10000, 200000) * scale / 24.0)) * 24)
        reqs.append((p, V, E, T, nk, steps, float(rng.exponential(1.0 / rate))))
    return reqs


def run_alone_timed(G, p, V, E, T, nk, steps):
    """one request on the plain path: create, set up, step, observables;
    host seconds with the device work waited for"""
    import numpy as np
    t = time.perf_counter()
    sim = G.Simulation(p)
    sim.init(V, E, T, nk)
    sim.step(steps)
    obs = sim.observables()
    sim.sync()
    dt = time.perf_counter() - t
    sim.close()
    return dt, bool(np.isfinite(obs[:6]).all())


def run_served(G, nreq=40, rate=2.0, scale=0.1, nthreads=8, schedule=None):
    """Poisson-arriving sweep requests admitted by the request server by
    device-memory footprint (served_requests), against the plain path: the
    same requests each run alone, and those alone times pushed through a
    one-at-a-time queue under the same arrival times.  `schedule`: a launch
    schedule (the batched leg's tuned one) applied to every admitted
    request.  The step counts are the configuration's 10k..200k times
    `scale`: at 0.1 the requests arriving at 2/s bring about twice the
    plain path's capacity in work, so requests queue as they do at the
    configuration's full step counts (which bring about twenty times); at
    0.02 the GPU would sit idle half the time and nothing would queue."""
    import numpy as np
    reqs = served_requests(G, nreq, rate, scale)
    srv = G.Server(nthreads=nthreads, round_steps=96)
    if schedule:
        srv.set_schedule(**schedule)
    t0 = srv.clock()
    for p, V, E, T, nk, steps, gap in reqs:
        time.sleep(gap)
        srv.submit(p, V, E, T, nk, steps)
    got = []
    while len(got) < nreq:
        more = srv.poll(64, wait=120.0)
        if not more:
            break
        got += more
    t1 = srv.clock()
    srv.close()
    by_id = {r["id"]: r for r in got}
    ids = sorted(by_id)
    lat = np.array([by_id[i]["t_end"] - by_id[i]["t_submit"] for i in ids])
    wait = np.array([by_id[i]["t_start"] - by_id[i]["t_submit"] for i in ids])
    service = np.array([by_id[i]["t_end"] - by_id[i]["t_start"] for i in ids])
    arrive = np.array([by_id[i]["t_submit"] for i in ids])
    ok = int(sum(r["status"] == 0 for r in got))
    statuses = {}
    for r in got:
        statuses[str(r["status"])] = statuses.get(str(r["status"]), 0) + 1
    work = sum(r["ns"] * r["steps"] for r in got if r["status"] == 0)
    # the plain path: every request alone, one after another
    alone, alone_ok = [], True
    for p, V, E, T, nk, steps, _ in reqs:
        dt, fin = run_alone_timed(G, p, V, E, T, nk, steps)
        alone.append(dt)
        alone_ok = alone_ok and fin
    alone = np.array(alone)
    # one at a time in arrival order under the same arrivals
    done, plain_lat = 0.0, []
    for a, d in zip(arrive, alone[:len(arrive)]):
        done = max(done, a) + d
        plain_lat.append(done - a)
    plain_lat = np.array(plain_lat)
    plain_span = done - arrive[0] if len(arrive) else float("nan")
    span = t1 - t0
    return {"metric": "served sweep requests", "requests": nreq, "completed": ok, "statuses": statuses,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "admission_wait_p50_s": float(np.percentile(wait, 50)),
            "service_p50_s": float(np.percentile(service, 50)),
            "sims_per_hour": 3600.0 * len(got) / span, "value": work / span, "unit": UNIT,
            "plain_alone_p50_s": float(np.percentile(alone, 50)), "plain_alone_p99_s": float(np.percentile(alone, 99)),
            "plain_p50_s": float(np.percentile(plain_lat, 50)), "plain_p99_s": float(np.percentile(plain_lat, 99)),
            "plain_sims_per_hour": 3600.0 * len(plain_lat) / plain_span,
            "plain_busy_s": float(alone.sum()), "plain_finite": alone_ok,
            "vs_plain": {"p50": float(np.percentile(lat, 50) / np.percentile(plain_lat, 50)),
                         "p99": float(np.percentile(lat, 99) / np.percentile(plain_lat, 99)),
                         "sims_per_hour": float((len(got) / span) / (len(plain_lat) / plain_span))},
            "plain_note": "each request alone on the plain path (create, set-up, steps, observables), then those "
                          "times pushed through a one-at-a-time queue under the same arrival times",
            "arrival_rate_per_s": rate, "step_scale": scale,
            "steps_per_request": [int(min(r[5] for r in reqs)), int(max(r[5] for r in reqs))],
            "dtype": "f32-bulk", "schedule": schedule or "default",
            "config": "Poisson arrivals at %g/s; kon log-U 1e-4..1e-1, koff log-U 1e-3..1e-1, knobs 50..1000, "
                      "walls/Lz 0.002..0.02, Lx 32..128, Ly = Lz 24..48, 600- or 2562-vertex mesh, "
                      "10k..200k steps x %g" % (rate, scale)}


def run_e2e(G, sim, st, steps, ns):
    """Same metric through the public API with host buffers: set_state of
    the full state `st` (the state the timed steps started from) from
    page-locked memory, the same `steps` steps each followed by the RBCdata
    record (vertex x,y,z,ix,iy,bondi) copied to page-locked host memory
    (queued behind the step), then the full state back.
    Host wall clock with a device synchronize on both ends."""
    import numpy as np
    pinned = {}
    for k, a in st.a.items():
        pa = G.PinnedArray(a.size, a.dtype)
        pa.array[:] = a
        pinned[k] = pa
        st.a[k] = pa.array
    # the RBCdata record of every step into page-locked host buffers
    # (alternating), queued behind the step without a host wait
    rec = [G.PinnedArray(sim.record_bytes(), np.uint8) for _ in range(2)]
    # the final state comes back into page-locked arrays the caller owns
    out = G.State(st.ns, st.nv, st.nlig, st.ncell, lcap=int(sim.L.irbc_llist_total(sim.h)) + (1 << 20))
    for k, a in out.a.items():
        pa = G.PinnedArray(a.size, a.dtype)
        pinned["out_" + k] = pa
        out.a[k] = pa.array
    h2d = sum(st.a[k].nbytes for k in st.a)
    d2h_rec = rec[0].array.nbytes
    sim.sync()
    t0 = time.perf_counter()
    sim.set_state(st)
    t1 = time.perf_counter()
    for k in range(steps):
        sim.step(1)
        sim.record_async(rec[k & 1])
    sim.sync()
    t2 = time.perf_counter()
    v = out.view()
    sim._ck(sim.L.irbc_get_state(sim.h, __import__("ctypes").byref(v)), "irbc_get_state")
    out.absorb(v)
    sim.sync()
    t3 = time.perf_counter()
    nv = sim.nv
    last = rec[(steps - 1) & 1].array
    assert np.array_equal(last[:8 * nv].view(np.float64), out.a["x"]), "record and state disagree"
    dt = t3 - t0
    # the list entries copied, not the buffer's spare room
    d2h = d2h_rec * steps + sum(out.a[k].nbytes for k in out.a if k != "lidx") + 4 * int(out.a["llen"].sum())
    return {"value": ns * steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d / steps),
            "d2h_bytes_per_step": int(d2h / steps),
            "seconds": {"set_state": t1 - t0, "steps": t2 - t1, "get_state": t3 - t2}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=780)
    ap.add_argument("--warmup", type=int, default=12)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-batch", dest="batch", action="store_false")
    ap.add_argument("--no-serve", dest="serve", action="store_false")
    # the batched or served leg alone (profiling runs)
    ap.add_argument("--batch-only", action="store_true")
    ap.add_argument("--serve-only", action="store_true")
    ap.add_argument("--batch-replicas", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=240)
    ap.add_argument("--serve-scale", type=float, default=0.1)
    args = ap.parse_args()
    # at least 3; and past the third collision, so the first 24-step graph
    # is captured before the timed steps
    args.warmup = max(args.warmup, 36)
    if args.impl == "reference":
        run_reference(args)
    elif args.batch_only:
        import irbc_b200 as G
        print(json.dumps({"batched": run_batched(G, nrep=args.batch_replicas, steps=args.batch_steps)}))
    elif args.serve_only:
        import irbc_b200 as G
        print(json.dumps({"served": run_served(G, scale=args.serve_scale)}))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
