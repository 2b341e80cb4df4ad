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
    # membrane, streams and graphs try two values each, chunk three; each
    # candidate runs once untimed and once timed, all feasible for this
    # 600-vertex mesh
    assert taken == (2 + 2 + 2 + 3) * 2 * 24
    assert sched == b.schedule()
    assert sched["streams"] in (1, 2) and sched["membrane"] in (1, 2) and sched["graphs"] in (0, 1)
    assert sched["chunk"] in (24, 96, 240)
    b.step(30)
    for s, p in zip(sims, params):
        assert H.compare(s.get_state(), _alone(p, V, E, T, 300, taken + 30), 0.0) == {}
    b.close()
    for s in sims:
        s.close()
