"""The large workload's membrane over a long run, on the GPU in FP64: the
2562-vertex discocyte (1000 knobs, SRD angle 130 deg, dtcd 0.025, walls/Lz
0.01, a 32^3 box with 40,000 solvent particles), as in
oracle/discocyte_stability.py, which runs the same setting in the oracle.

With the WLC persistence constant scaled to the mesh (the workload's
elap) the cell stays physical for 50,000 steps: finite, healthy, area and
volume within a few percent of their set-up values.  With the constant
the reference hard-codes for its 0.98-edge mesh (0.0005) the cell blows
up, and the health check reports it."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(elap, seed=31):
    import irbc_b200 as G
    from irbc_b200 import mesh
    V, E, T = mesh.discocyte()
    a = math.radians(130.0)
    p = G.default_params(Lx=32.0, Ly=32.0, Lz=32.0, Ns=40000, Nt=len(V), dtcd=0.025, walls=0.32,
                         cosalpha=math.cos(a), sinalpha=math.sin(a), onrate=0.005, offrate=0.015, elap=elap,
                         seed=seed)
    sim = G.Simulation(p)
    sim.init(V, E, T, 1000)
    return G, sim


def test_discocyte_runs_50k_steps_with_the_scaled_persistence_constant():
    from irbc_b200 import mesh
    V, E, _ = mesh.discocyte()
    G, sim = _sim(mesh.scaled_elap(V, E))
    S0, V0 = sim.report()[2], sim.report()[3]
    rows = []
    for k in range(10):
        sim.step(5000)
        sim.sync()
        assert sim.health() == 0, (k, sim.health())
        ob = sim.observables()
        st = sim.get_state(solvent=False, llist=False)
        vmax = float(np.sqrt(st.a["vx"] ** 2 + st.a["vy"] ** 2 + st.a["vz"] ** 2).max())
        rows.append((ob[4] / S0, ob[5] / V0, vmax))
        assert np.isfinite(ob[:9]).all()
        assert 0.93 < ob[4] / S0 < 1.01, rows
        assert 0.95 < ob[5] / V0 < 1.05, rows
        assert vmax < 10.0, rows
    sim.close()


def test_the_literal_persistence_constant_blows_up_and_is_reported():
    from irbc_b200 import mesh
    G, sim = _sim(mesh.REF_ELAP)
    rc = 0
    for k in range(40):
        sim.L.irbc_step(sim.h, 100)
        rc = sim.L.irbc_sync(sim.h)
        if rc:
            break
    assert rc == G.ERR_HEALTH, rc
    assert sim.health() & G.HEALTH_MEMBRANE
    sim.close()
