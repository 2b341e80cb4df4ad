"""Batches and the request server: a simulation computes the same thing
alone, in a batch, or admitted by the server in a mix with others (bit for
bit: each keeps its own streams, memory and draw epochs)."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _small(seed, ns=20000, precision=0, **over):
    op, orc = H.make_oracle(ns=ns, seed=seed, **over)
    import irbc_b200 as G
    p = H.to_irbc_params(op, seed, precision)
    return op, p


def _run_alone(p, V, E, T, nknobs, steps):
    import irbc_b200 as G
    sim = G.Simulation(p)
    sim.init(V, E, T, nknobs)
    sim.step(steps)
    st = sim.get_state()
    sim.close()
    return st


def test_batch_equals_members_alone():
    import irbc_b200 as G
    V, E, T = H.troph()
    cfgs = [(3, 0, {}), (4, 1, {}), (5, 0, dict(onrate=300.0, offrate=50.0))]
    sims, params = [], []
    for seed, prec, over in cfgs:
        _, p = _small(seed, precision=prec, **over)
        s = G.Simulation(p)
        s.init(V, E, T, 300)
        sims.append(s)
        params.append(p)
    b = G.Batch(nthreads=2)
    for s in sims:
        b.add(s)
    b.step(37)
    b.step(60)
    for s, p in zip(sims, params):
        ref = _run_alone(p, V, E, T, 300, 97)
        assert H.compare(s.get_state(), ref, 0.0) == {}
    b.close()
    for s in sims:
        s.close()


def test_server_results_same_alone_and_in_mix():
    """Six requests with different seeds, rates, precisions and lengths;
    a budget for two at a time, so later ones wait for memory and join as
    earlier ones finish.  Every kept result equals the same request run
    alone, and at most two ran at once."""
    import irbc_b200 as G
    V, E, T = H.troph()
    reqs = []
    for k in range(6):
        seed = 20 + k
        _, p = _small(seed, precision=k % 2, onrate=0.005 * (k + 1), offrate=0.015)
        reqs.append((p, 100 + 20 * k, 48 + 24 * k))
    fp = max(G.lib().irbc_footprint_bytes(G.C.byref(p), len(V), len(E), len(T)) for p, _, _ in reqs)
    srv = G.Server(budget_bytes=int(2.5 * fp), nthreads=2, round_steps=24)
    ids = {}
    spans = []

    def check(results):
        # each kept result stays charged to the budget until it is handed
        # back: compare it with the request run alone, then release it
        for r in results:
            assert r["status"] == 0
            p, nk, steps = ids[r["id"]]
            assert r["steps"] == steps
            assert r["t_submit"] <= r["t_start"] <= r["t_end"]
            spans.append((r["t_start"], r["t_end"]))
            ref = _run_alone(p, V, E, T, nk, steps)
            assert H.compare(r["sim"].get_state(), ref, 0.0) == {}, r["id"]
            r["sim"].close()
        return len(results)

    for p, nk, steps in reqs[:3]:
        ids[srv.submit(p, V, E, T, nk, steps, keep=True)] = (p, nk, steps)
    got = check(srv.poll(8, wait=30.0))
    for p, nk, steps in reqs[3:]:
        ids[srv.submit(p, V, E, T, nk, steps, keep=True)] = (p, nk, steps)
    while got < len(reqs):
        more = srv.poll(8, wait=60.0)
        assert more, "server stalled"
        got += check(more)
    st = srv.status()
    assert st["used"] == 0 and st["active"] == 0, st
    # never more than two admitted at the same time
    for t, _ in spans:
        assert sum(1 for a, b in spans if a <= t < b) <= 2
    srv.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_one_stream_equals_two(precision):
    """irbc_set_streams(1) puts the membrane kernels on the solvent's stream:
    the same state, bit for bit, across collisions and a list update."""
    import irbc_b200 as G
    V, E, T = H.troph()
    _, p = _small(9, precision=precision, onrate=300.0, offrate=50.0)
    a = G.Simulation(p)
    a.init(V, E, T, 300)
    a.set_streams(1)
    a.step(50)
    a.set_streams(2)
    a.step(47)
    ref = _run_alone(p, V, E, T, 300, 97)
    assert H.compare(a.get_state(), ref, 0.0) == {}
    a.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_one_block_membrane_equals_wide_kernels(precision):
    """The one-block membrane step (an option for meshes up to 1024
    vertices, such as this 600-vertex one) and the wide kernels (the
    default) give the same state, bit for bit, across collisions, bond
    events and a list update."""
    import irbc_b200 as G
    V, E, T = H.troph()
    _, p = _small(13, precision=precision, onrate=300.0, offrate=50.0)
    out = []
    for mode in (1, 2):
        s = G.Simulation(p)
        s.init(V, E, T, 300)
        s.set_membrane_kernels(mode)
        s.step(97)
        out.append(s.get_state())
        s.close()
    assert H.compare(out[0], out[1], 0.0) == {}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("which", ["troph", "disc"])
def test_cluster_membrane_equals_wide_kernels(precision, which):
    """The membrane step as one launch of a thread-block cluster (any mesh:
    the 600-vertex trophozoite and the 2562-vertex discocyte) and the wide
    kernels give the same state, bit for bit, across collisions, bond
    events, list updates and captured graphs."""
    import irbc_b200 as G
    from irbc_b200 import mesh
    if which == "troph":
        V, E, T = H.troph()
        _, p = _small(14, precision=precision, onrate=300.0, offrate=50.0)
        nk = 300
    else:
        V, E, T = mesh.discocyte()
        _, p = _small(15, precision=precision, onrate=300.0, offrate=50.0)
        p.Nt, p.elap, nk = len(V), mesh.scaled_elap(V, E), 900
    out = []
    for mode, graphs in ((1, 0), (3, 0), (3, 1)):
        s = G.Simulation(p)
        s.init(V, E, T, nk)
        s.set_membrane_kernels(mode)
        s.set_graphs(graphs)
        s.step(97)
        s.step(80)
        out.append(s.get_state())
        s.close()
    assert H.compare(out[1], out[0], 0.0) == {}
    assert H.compare(out[2], out[0], 0.0) == {}


def test_server_reports_a_failed_set_up_alone():
    """A request whose set-up fails on the server's set-up thread (a knob
    count above the mesh's vertex count: irbc_init rejects it) ends with
    that error and gives its memory back; the requests around it finish and
    equal themselves run alone."""
    import irbc_b200 as G
    V, E, T = H.troph()
    nv = len(V) // 3 if np.ndim(V) == 1 else len(V)
    reqs = []
    for k in range(3):
        _, p = _small(70 + k, precision=k % 2)
        reqs.append((p, nv + 1 if k == 1 else 200, 72))
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
        if nk > nv:
            assert r["status"] == G.ERR_ARG and r["sim"] is None
            continue
        assert r["status"] == 0
        ref = _run_alone(p, V, E, T, nk, steps)
        assert H.compare(r["sim"].get_state(), ref, 0.0) == {}
        r["sim"].close()
    st = srv.status()
    assert st["used"] == 0 and st["active"] == 0, st
    srv.close()
