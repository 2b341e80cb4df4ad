"""The benchmarked workload at its full size against the oracle: box
128 x 64 x 64 with 5,242,880 solvent particles, the 2562-vertex discocyte
with 1000 knobs, SRD angle 130 deg, dtcd 0.025, walls 0.64
(irbc_b200.workloads.large_params; bond rates raised so that bonds form and
break).  The GPU sets the simulation up; the oracle takes that state and
mesh, and both advance step by step, each half-step started from the
oracle's state (maincode.cpp:461-764).  The 25 steps hold two collisions,
the second of which is the library's 16th and re-sorts the solvent
physically by cell, and a triangle-list update (llistupdate) on the
full-size lists.

FP64 tolerance: positions, velocities and forces within 1e-12 normwise
relative error; cell indices, lists, bond states, image counters and
ligand occupancy exact."""
import pytest

import helpers as H

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def test_large_workload_full_size_step_by_step():
    import irbc_b200 as G
    from irbc_b200 import workloads
    p = workloads.large_params(seed=1234, precision=0, onrate=300.0, offrate=50.0)
    V, E, T = workloads.large_mesh()
    sim = G.Simulation(p)
    sim.init(V, E, T, workloads.LARGE["nknobs"])
    start = sim.get_state()
    assert start.ns == 5242880 and start.nv == 2562
    # 14 collisions first (their results are discarded): the collision at
    # step 24 below is then the library's 16th, which re-sorts the arrays
    for k in range(14):
        sim.call("collide", k)
    # the list update falls at step 5 (the counter runs to uplist = 390)
    start.s["upd"] = int(0.5 / (p.walls * p.dtmd)) - 6
    sim.set_state(start)
    op, orc = H.oracle_like(sim, p)
    bonds = 0
    for k in range(25):
        sim.set_state(G.State.from_other(orc.get_state()))
        sim.call("step_part1")
        orc.step_part1()
        assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}, ("part1", k)
        sim.call("step_part2")
        orc.step_part2()
        ref = orc.get_state()
        assert H.compare(sim.get_state(), ref, RTOL) == {}, ("part2", k)
        bonds = max(bonds, int(ref.a["bondi"].sum()))
    assert ref.s["step"] == 25 and bonds > 0
    sim.close()
