"""The run-time health check: the streaming and membrane kernels raise bits
of a health word when a particle or vertex goes non-finite (or a particle
leaves the box), and the host turns the word into IRBC_ERR_HEALTH.  The
reference has no such check (a blown-up run of it keeps writing NaN into
RBCdata.dat).  The bad values are planted in a host-side copy of a healthy
state and loaded with irbc_set_state; NaN only travels through arithmetic
and comparisons, never into an index (every float-to-cell conversion is
bounds-checked, and NaN converts to 0)."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _sim(seed=41, precision=0, **over):
    import irbc_b200 as G
    op, orc = H.make_oracle(ns=20000, seed=seed, **over)
    sim = H.gpu_like(op, orc, seed, precision)
    return G, op, orc, sim


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_solvent_particle_is_reported(precision):
    G, op, orc, sim = _sim(precision=precision)
    sim.step(15)  # across a collision
    sim.sync()
    assert sim.health() == 0
    good = sim.get_state()
    bad = good.copy()
    k = int(np.argmax(bad.a["sz"] > 20.0))  # a particle far from the membrane and the walls
    bad.a["svx"][k] = np.nan
    sim.set_state(bad)
    assert sim.health() == 0  # set_state starts a fresh state
    sim.step(2)
    rc = sim.L.irbc_sync(sim.h)
    assert rc == G.ERR_HEALTH
    assert "solvent" in sim.L.irbc_last_error(sim.h).decode()
    assert sim.health() & G.HEALTH_SOLVENT
    # a simulation found unhealthy is not stepped further
    assert sim.L.irbc_step(sim.h, 1) == G.ERR_HEALTH
    # a healthy state clears it
    sim.set_state(good)
    sim.step(3)
    sim.sync()
    assert sim.health() == 0
    sim.close()


def test_nan_vertex_is_reported():
    G, op, orc, sim = _sim(seed=43)
    sim.step(4)
    bad = sim.get_state()
    bad.a["vy"][7] = np.inf
    sim.set_state(bad)
    sim.step(2)
    assert sim.L.irbc_sync(sim.h) == G.ERR_HEALTH
    assert sim.health() & G.HEALTH_MEMBRANE
    sim.close()


def test_server_retires_only_the_unhealthy_request():
    """Three requests, one of which has a zero vertex mass (its membrane
    velocities are not finite from the first half-kick): that one ends with
    IRBC_ERR_HEALTH, the other two finish and equal themselves run alone."""
    import irbc_b200 as G
    V, E, T = H.troph()
    reqs = []
    for k in range(3):
        op, _ = H.make_oracle(ns=20000, seed=60 + k)
        p = H.to_irbc_params(op, 60 + k, 0)
        if k == 1:
            p.pmass = 0.0
        reqs.append((p, 200, 96))
    srv = G.Server(nthreads=2, round_steps=24)
    ids = {}
    for p, nk, steps in reqs:
        ids[srv.submit(p, V, E, T, nk, steps, keep=True)] = (p, nk, steps)
    got = []
    while len(got) < len(reqs):
        more = srv.poll(8, wait=60.0)
        assert more, "server stalled"
        got += more
    for r in got:
        p, nk, steps = ids[r["id"]]
        if p.pmass == 0.0:
            assert r["status"] == G.ERR_HEALTH and r["sim"] is None
            continue
        assert r["status"] == 0
        assert r["steps"] == steps
        sim = G.Simulation(p)
        sim.init(V, E, T, nk)
        sim.step(steps)
        assert H.compare(r["sim"].get_state(), sim.get_state(), 0.0) == {}
        sim.close()
        r["sim"].close()
    st = srv.status()
    assert st["used"] == 0 and st["active"] == 0, st
    srv.close()
