"""irbc_batch_autotune times candidate launch schedules on the batch's own
members, so its trial steps are real steps.  No schedule field changes what
a member computes: after tuning and further steps under the chosen
schedule, every member equals the same simulation run alone for as many
steps, bit for bit."""
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _params(seed, precision, onrate=0.005, offrate=0.015):
    import oracle as O
    op = O.default_params(Ns=20000, onrate=onrate, offrate=offrate)
    return H.to_irbc_params(op, seed, precision)


def _alone(p, V, E, T, nknobs, steps):
    import irbc_b200 as G
    sim = G.Simulation(p)
    sim.init(V, E, T, nknobs)
    sim.step(steps)
    st = sim.get_state()
    sim.close()
    return st


def test_autotuned_batch_equals_members_alone():
    import irbc_b200 as G
    V, E, T = H.troph()
    params = [_params(41, 0), _params(42, 1, onrate=300.0, offrate=50.0)]
    sims = []
    b = G.Batch(nthreads=2)
    for p in params:
        s = G.Simulation(p)
        s.init(V, E, T, 300)
        sims.append(s)
        b.add(s)
    sched, taken = b.autotune(trial_steps=24, repeats=1)
    # fused, membrane, streams and graphs try two values each, chunk three;
    # each candidate runs once untimed and once timed, all feasible for
    # this 600-vertex mesh
    assert taken == (2 + 2 + 2 + 2 + 3) * 2 * 24
    assert sched == b.schedule()
    assert sched["streams"] in (1, 2) and sched["membrane"] in (1, 2) and sched["graphs"] in (0, 1)
    assert sched["chunk"] in (24, 96, 240)
    b.step(30)
    for s, p in zip(sims, params):
        assert H.compare(s.get_state(), _alone(p, V, E, T, 300, taken + 30), 0.0) == {}
    b.close()
    for s in sims:
        s.close()


def test_server_schedule_keeps_results():
    """A server given a launch schedule applies it to every request it
    admits; the one-block membrane form only where the mesh fits it (the
    600-vertex mesh), the wide kernels elsewhere (the 2562-vertex
    discocyte).  Every kept result equals the same request run alone."""
    import irbc_b200 as G
    from irbc_b200 import mesh
    troph, disc = H.troph(), mesh.discocyte()
    reqs = [(_params(51, 0), troph, 96), (_params(52, 1, onrate=300.0, offrate=50.0), troph, 120),
            (_params(53, 1), disc, 72)]
    fp = sum(G.lib().irbc_footprint_bytes(G.C.byref(p), len(m[0]), len(m[1]), len(m[2])) for p, m, _ in reqs)
    srv = G.Server(budget_bytes=int(1.5 * fp), nthreads=2, round_steps=24)
    srv.set_schedule(streams=1, membrane=2, graphs=1, chunk=48)
    ids = {}
    for p, (V, E, T), steps in reqs:
        ids[srv.submit(p, V, E, T, 300, steps, keep=True)] = (p, (V, E, T), steps)
    got = []
    while len(got) < len(reqs):
        more = srv.poll(8, wait=60.0)
        assert more, "server stalled"
        got += more
    for r in got:
        assert r["status"] == 0
        p, (V, E, T), steps = ids[r["id"]]
        assert H.compare(r["sim"].get_state(), _alone(p, V, E, T, 300, steps), 0.0) == {}, r["id"]
        r["sim"].close()
    srv.close()
