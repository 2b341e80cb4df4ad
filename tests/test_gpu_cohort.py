"""Cohorts: FP32 simulations stepped together with one kernel launch per
phase of the step (irbc_schedule.fused), each launch's blocks split among
the members.  Every member must end bit for bit where the same simulation
ends alone on the plain path: uneven boxes, knob counts and bond rates,
two meshes in one cohort, list updates and the physical re-sort inside the
stretch, and members that fall out of phase with the others."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _params(seed, Lx, ns, precision=1, **over):
    import irbc_b200 as G
    p = G.default_params(Lx=float(Lx), Ns=ns, seed=seed, precision=precision, **over)
    return p


def _alone(p, V, E, T, nknobs, steps):
    import irbc_b200 as G
    sim = G.Simulation(p)
    sim.init(V, E, T, nknobs)
    sim.step(steps)
    st = sim.get_state()
    sim.close()
    return st


def _check(sims, cfgs, steps):
    for sim, (p, (V, E, T), nk) in zip(sims, cfgs):
        ref = _alone(p, V, E, T, nk, steps)
        bad = H.compare(sim.get_state(), ref, 0.0)
        assert bad == {}, (p.seed, bad)


def test_fused_batch_equals_members_alone():
    """Five FP32 members (boxes 40..72 long, 300..600 knobs, one with bond
    rates raised so that bonds form and break) stepped 200 steps as one
    cohort, in two calls: 16 collisions (the 16th re-sorts the solvent),
    and list updates at steps 82 and 165."""
    import irbc_b200 as G
    troph = H.troph()
    cfgs = []
    for r, (Lx, nk, over) in enumerate([(60, 500, {}), (40, 300, {}), (72, 600, dict(onrate=300.0, offrate=50.0)),
                                        (48, 400, {}), (56, 350, {})]):
        cfgs.append((_params(700 + r, Lx, int(Lx * 40 * 41 * 3), **over), troph, nk))
    sims = []
    b = G.Batch(nthreads=2)
    assert b.schedule()["fused"] == 1
    for p, (V, E, T), nk in cfgs:
        s = G.Simulation(p)
        s.init(V, E, T, nk)
        sims.append(s)
        b.add(s)
    launches0 = sims[0].launch_count()
    b.step(37)
    b.step(163)
    # one launch per phase: far fewer than five members' own launches
    assert sims[0].launch_count() - launches0 < 200 * 40
    _check(sims, cfgs, 200)
    b.close()
    for s in sims:
        s.close()


def test_fused_cohort_with_two_meshes_and_an_fp64_member():
    """The 600-vertex trophozoite and the 2562-vertex discocyte in one
    cohort, and an FP64 member beside it (stepped by the pool of host
    threads): each equals itself alone."""
    import irbc_b200 as G
    from irbc_b200 import mesh
    troph, disc = H.troph(), mesh.discocyte()
    de = mesh.scaled_elap(disc[0], disc[1])
    cfgs = [(_params(801, 48, 48 * 40 * 41 * 3), troph, 300),
            (_params(802, 40, 40 * 40 * 41 * 3, Nt=len(disc[0]), elap=de, walls=0.4), disc, 800),
            (_params(803, 44, 44 * 40 * 41 * 3, precision=0), troph, 250)]
    sims = []
    b = G.Batch(nthreads=2)
    for p, (V, E, T), nk in cfgs:
        s = G.Simulation(p)
        s.init(V, E, T, nk)
        sims.append(s)
        b.add(s)
    b.step(60)
    b.step(36)
    _check(sims, cfgs, 96)
    b.close()
    for s in sims:
        s.close()


def test_members_out_of_phase_form_their_own_cohorts():
    """A member that has taken 7 steps alone before joining is out of phase
    with the others (its collisions fall on other steps): the batch steps
    it in a cohort of its own, and every member still equals itself alone."""
    import irbc_b200 as G
    troph = H.troph()
    cfgs = [(_params(900 + r, 40 + 4 * r, (40 + 4 * r) * 40 * 41 * 3), troph, 300) for r in range(3)]
    sims = []
    for p, (V, E, T), nk in cfgs:
        s = G.Simulation(p)
        s.init(V, E, T, nk)
        sims.append(s)
    sims[2].step(7)
    b = G.Batch(nthreads=2)
    for s in sims:
        b.add(s)
    b.step(50)
    _check(sims[:2], cfgs[:2], 50)
    _check(sims[2:], cfgs[2:], 57)
    b.close()
    for s in sims:
        s.close()
