"""CUDA library against the CPU oracle on the same seeded inputs.

FP64 tolerance: positions, velocities and forces within 1e-12 normwise
relative error (max|gpu - oracle| / max|oracle| per field); cell indices,
llist entries, bond states, image counters and ligand occupancy exact."""
import numpy as np
import pytest

import oracle as O
import helpers as H

pytestmark = pytest.mark.gpu
RTOL = 1e-12


@pytest.fixture(scope="module")
def base():
    """Oracle after set-up and 25 steps with raised bond rates (so bonds
    exist and two collisions have happened)."""
    op, orc = H.make_oracle(ns=40000, seed=11, onrate=300.0, offrate=50.0)
    orc.step(25)
    return op, orc.get_mesh(), orc.get_state()


def fresh_oracle(op, mesh, st, seed=11):
    o = O.Oracle(op, seed)
    o.set_mesh(mesh)
    o.set_state(st)
    return o


def test_init_matches_oracle():
    op, orc = H.make_oracle(ns=40000, seed=5)
    import irbc_b200 as G
    sim = G.Simulation(H.to_irbc_params(op, 5))
    V, E, T = H.troph()
    sim.init(V, E, T, 500)
    np.testing.assert_array_equal(sim.report(), orc.report())
    a, s = sim.get_mesh_arrays()
    M = orc.get_mesh()
    for k in ("e1", "e2", "es1", "es2", "iedge", "t1", "t2", "t3", "l0", "kappap", "tarea"):
        np.testing.assert_array_equal(a[k], M.a[k], err_msg=k)
    assert s["Sarea0"] == M.s["Sarea0"] and s["Volume0"] == M.s["Volume0"] and s["theta0"] == M.s["theta0"]
    bad = H.compare(sim.get_state(), orc.get_state(), RTOL)
    assert bad == {}


@pytest.mark.parametrize("phase", ["collide", "llist_update", "stream", "total_va", "pfdt", "forces"])
def test_phase_matches_oracle(base, phase):
    op, mesh, st = base
    o = fresh_oracle(op, mesh, st)
    sim = H.gpu_like(op, o, 11, state=st)
    if phase == "collide":
        sim.call("collide", 30)
        o.collide(30)
    else:
        sim.call(phase)
        getattr(o, phase)()
    g, r = sim.get_state(), o.get_state()
    bad = H.compare(g, r, RTOL)
    assert bad == {}, (phase, bad)


def test_collide_counts_every_particle_once(base):
    op, mesh, st = base
    o = fresh_oracle(op, mesh, st)
    sim = H.gpu_like(op, o, 11, state=st)
    sim.call("collide", 40)
    g = sim.get_state()
    counts = np.bincount(g.a["spid"], minlength=sim.ncell)
    assert counts.sum() == st.ns
    # momentum of the solvent+membrane changes only by the ghost terms:
    # check the energy stays finite and the ids survive the counting sort
    assert np.isfinite(g.a["svx"]).all()


def test_steps_match_oracle(base):
    """30 full steps (three collisions, bonds at raised rates)."""
    op, mesh, st = base
    o = fresh_oracle(op, mesh, st)
    sim = H.gpu_like(op, o, 11, state=st)
    for k in range(30):
        sim.call("step_part1")
        o.step_part1()
        g, r = sim.get_state(), o.get_state()
        assert H.compare(g, r, RTOL) == {}, ("part1", k)
        sim.call("step_part2")
        o.step_part2()
    g, r = sim.get_state(), o.get_state()
    assert H.compare(g, r, RTOL) == {}
    assert g.s["step"] == r.s["step"]


def test_llist_update_step_and_stale_tail():
    """Run through the llist update at step 82 (uplist = 83)."""
    op, orc = H.make_oracle(ns=20000, seed=21)
    orc.step(80)
    st = orc.get_state()
    sim = H.gpu_like(op, orc, 21, state=st)
    for k in range(6):
        sim.call("step_part1"); orc.step_part1()
        sim.call("step_part2"); orc.step_part2()
    assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}


def test_full_size_config1_init_and_steps():
    """define.h sizes (Ns = 960000): set-up and 12 steps incl. a collision."""
    op, orc = H.make_oracle(ns=960000, seed=3)
    import irbc_b200 as G
    sim = G.Simulation(H.to_irbc_params(op, 3))
    V, E, T = H.troph()
    sim.init(V, E, T, 500)
    assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}
    sim.step(12)
    orc.step(12)
    assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}
