"""The CUDA library against the oracle on the large workload's membrane:
the 2562-vertex discocyte with 1000 knobs, SRD angle 130 deg, dtcd 0.025
and walls/Lz 0.01, in a 32^3 box with a thin solvent.  The oracle itself
equals the reference bit for bit on this mesh (test_oracle_vs_ref.py).

FP64 tolerance: positions, velocities and forces within 1e-12 normwise
relative error; cell indices, bond states, image counters and ligand
occupancy exact."""
import math

import pytest

import oracle as O
import helpers as H

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def test_discocyte_steps_match_oracle_step_by_step():
    """24 steps (two collisions, bonds at raised rates), each started from
    the oracle's state: part 1 and part 2 within 1e-12."""
    import irbc_b200 as G
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte()
    a = math.radians(130.0)
    op = O.default_params(Lx=32.0, Ly=32.0, Lz=32.0, Ns=10000, Nt=len(V), dtcd=0.025, walls=0.32,
                          cosalpha=math.cos(a), sinalpha=math.sin(a), onrate=300.0, offrate=50.0)
    orc = O.Oracle(op, 31)
    orc.init(V, E, T, 1000)
    sim = H.gpu_like(op, orc, 31)
    for k in range(24):
        sim.set_state(G.State.from_other(orc.get_state()))
        sim.call("step_part1")
        orc.step_part1()
        assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}, ("part1", k)
        sim.call("step_part2")
        orc.step_part2()
        assert H.compare(sim.get_state(), orc.get_state(), RTOL) == {}, ("part2", k)
    assert int(orc.get_state().a["bondi"].sum()) > 0
    sim.close()
