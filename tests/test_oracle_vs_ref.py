"""The CPU oracle against the reference compiled from its own sources.

The reference's main() runs unchanged (oracle/ref_hooks.cpp), fed the same
counter draw stream as the oracle.  Both are built with IEEE double and no
FMA contraction, so every field must agree bit for bit.  Skipped where the
reference build (oracle/_ref) is absent.
"""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not os.path.exists(O.ref_lib_path("small")),
                                reason="reference build oracle/_ref/small not present")


def _run_ref(stop, seed, want, **kw):
    R = O.Reference("small")
    snaps = {}

    def cb(s):
        if s in want:
            snaps[s] = R.get_state(s)
    vf, ef, tf = O.troph_files()
    assert R.run(vf, ef, tf, 500, stop, seed=seed, on_step=cb, **kw) == 0
    return R, snaps


def _diff(a, b):
    d = O.compare_states(a, b)
    return {k: v for k, v in d.items() if v != 0}


def _crossing_state(st, M, ntri, seed):
    """A copy of st whose first 2*ntri particles sit 0.004 off the
    centroids of ntri sampled triangles, one on each side, moving at speed 5
    towards the membrane: each crosses it within dtmd (0.002).  Each one's
    indio names the side it starts on as the reference's side test reads
    it (1 where (B-A) x (C-A) points at the particle), so that none is
    skipped as already being on the wrong side."""
    out = st.copy()
    pos = np.stack([st.a["x"], st.a["y"], st.a["z"]], axis=1)
    T = np.stack([M.a["t1"], M.a["t2"], M.a["t3"]], axis=1)
    rng = np.random.default_rng(seed)
    for k, j in enumerate(rng.choice(len(T), ntri, replace=False)):
        A, B, C = pos[T[j]]
        c = (A + B + C) / 3.0
        n = np.cross(B - A, C - A)
        n /= np.linalg.norm(n)
        for side, i in ((1.0, 2 * k), (-1.0, 2 * k + 1)):
            out.a["sx"][i], out.a["sy"][i], out.a["sz"][i] = c + side * 0.004 * n
            out.a["svx"][i], out.a["svy"][i], out.a["svz"][i] = -side * 5.0 * n
            out.a["sindio"][i] = 1 if side > 0 else 0
    return out


def _check_crossings(R, orc, st, M, ntri, step):
    """reflectionFed on particles that must cross the membrane: the same
    contact times and the same reflected states."""
    cs = _crossing_state(st, M, ntri, 17)
    R.set_state(cs)
    orc.set_state(cs)
    fr = np.array([R.call_reflection(i) for i in range(2 * ntri)])
    fo = np.array([orc.reflection(i) for i in range(2 * ntri)])
    assert np.array_equal(fr, fo)
    # nearly all of them crossed (one may meet its triangle's edge or miss
    # its cell's list; both sides must agree on those too)
    assert np.count_nonzero(fr) >= 0.95 * 2 * ntri
    assert _diff(R.get_state(step), orc.get_state()) == {}
    assert _diff(R.get_state(step), cs) != {}  # and was reflected


def test_init_prints_known_answers(capfd):
    """maincode.cpp:256-257,345-346,366-368,446 printouts (seed-independent)."""
    R, _ = _run_ref(0, 7, set())
    out = capfd.readouterr().out
    for line in ("Mean edge is:\t0.983753", "Standard deviation is:\t0.0948865", "Sarea:\t501.17",
                 "Volume:\t840.892", "Shear modulus::\t1200", "Young's modulus::\t4711.11",
                 "Poisson's ratio::\t0.962963", "no of vertices selected:\t500"):
        assert line in out
    orc = O.Oracle(R.p, 7)
    V, E, T = O.load_mesh_files(*O.troph_files())
    orc.init(V, E, T, 500)
    rep = orc.report()
    np.testing.assert_allclose(rep[:8], [0.983753, 0.0948865, 501.17, 840.892, 1200, 4711.11, 0.962963, 500],
                               rtol=5e-6)


def test_oracle_init_and_steps_bit_exact():
    """Oracle set-up + 119 steps (12 collisions, one llist update at step 82,
    bonds forming and breaking at raised rates) equal the reference."""
    want = {0, 9, 10, 40, 81, 82, 83, 119}
    R, snaps = _run_ref(119, 99, want, onrate=300.0, offrate=50.0)
    V, E, T = O.load_mesh_files(*O.troph_files())
    orc = O.Oracle(R.p, 99)
    orc.init(V, E, T, 500)
    orc.step_part1()
    assert _diff(orc.get_state(), snaps[0]) == {}
    M, M2 = R.get_mesh(), orc.get_mesh()
    for k in M.a:
        assert np.array_equal(M.a[k], M2.a[k]), k
    orc.step_part2()
    bonds_seen = set()
    for s in range(1, 120):
        orc.step_part1()
        if s in snaps:
            st = orc.get_state()
            assert _diff(st, snaps[s]) == {}, s
            bonds_seen.add(int(st.a["bondi"].sum()))
            assert st.s["Sarea"] == snaps[s].s["Sarea"] and st.s["Volume"] == snaps[s].s["Volume"]
            assert np.array_equal(st.s["paraV"], snaps[s].s["paraV"])
        orc.step_part2()
    assert max(bonds_seen) > 0


def test_phase_functions_bit_exact():
    """Each reference function called directly on the same state."""
    R, snaps = _run_ref(30, 5, {19, 30}, onrate=300.0, offrate=50.0)
    st = snaps[30]
    M = R.get_mesh()
    orc = O.Oracle(R.p, 5)
    orc.set_mesh(M)
    for name, call_ref, call_orc in (
            ("collide", lambda: R.call_collide(31), lambda: orc.collide(31)),
            ("llist", R.call_llist, orc.llist_update),
            ("totalva", R.call_totalva, orc.total_va),
            ("pfdt", R.call_pfdt, orc.pfdt),
            ("forces", R.call_forces, orc.forces)):
        R.set_state(st)
        orc.set_state(st)
        call_ref()
        call_orc()
        a, b = R.get_state(30), orc.get_state()
        assert _diff(a, b) == {}, name
        assert a.s["Sarea"] == b.s["Sarea"], name
    # reflectionFed for every particle with a non-empty cell list
    R.set_state(st)
    orc.set_state(st)
    fr = np.array([R.call_reflection(i) for i in range(st.ns)])
    fo = np.array([orc.reflection(i) for i in range(st.ns)])
    assert np.array_equal(fr, fo)
    assert _diff(R.get_state(30), orc.get_state()) == {}
    _check_crossings(R, orc, st, M, 200, 30)


def test_cubic_solver_matches_reference():
    R = O.Reference("small")
    rng = np.random.default_rng(3)
    L = O.liboracle()
    xs_r, xs_o = np.zeros(3), np.zeros(3)
    for _ in range(2000):
        a, b, c = rng.normal(size=3) * rng.choice([1e-3, 1, 1e3, 1e6])
        nr = R.call_solvep3(xs_r.ctypes.data_as(O.D), a, b, c)
        no = L.orc_solve_p3(xs_o.ctypes.data_as(O.D), a, b, c)
        assert nr == no
        assert np.array_equal(xs_r[:nr if nr > 1 else 3], xs_o[:nr if nr > 1 else 3])
        assert R.call_solve(a, b, c) == L.orc_solve_cubic(a, b, c) or (
            np.isnan(R.call_solve(a, b, c)) and np.isnan(L.orc_solve_cubic(a, b, c)))


@pytest.mark.skipif(not os.path.exists(O.ref_lib_path("disc_small")),
                    reason="reference build oracle/_ref/disc_small not present")
def test_oracle_bit_exact_on_the_discocyte(tmp_path):
    """The large workload's membrane: the 2562-vertex discocyte written in the
    reference's file format, 1000 knobs, its SRD angle, dtcd and wall speed
    (a 32^3 box, thin solvent).  Mesh build, set-up and 89 steps (9
    collisions, the list update at step 82, bonds forming and breaking at
    raised rates) equal the reference bit for bit."""
    from irbc_b200 import mesh
    files = mesh.write_reference_files(str(tmp_path), *mesh.discocyte())
    want = {0, 10, 40, 82, 83, 89}
    R = O.Reference("disc_small")
    snaps = {}

    def cb(s):
        if s in want:
            snaps[s] = R.get_state(s)
    assert R.run(*files, 1000, 89, seed=31, on_step=cb, onrate=300.0, offrate=50.0) == 0
    assert R.p.Nt == 2562
    V, E, T = O.load_mesh_files(*files)
    orc = O.Oracle(R.p, 31)
    orc.init(V, E, T, 1000)
    M, M2 = R.get_mesh(), orc.get_mesh()
    for k in M.a:
        assert np.array_equal(M.a[k], M2.a[k]), k
    bonds_seen = set()
    for s in range(0, 90):
        orc.step_part1()
        if s in snaps:
            st = orc.get_state()
            assert _diff(st, snaps[s]) == {}, s
            assert st.s["Sarea"] == snaps[s].s["Sarea"] and st.s["Volume"] == snaps[s].s["Volume"]
            bonds_seen.add(int(st.a["bondi"].sum()))
        orc.step_part2()
    assert max(bonds_seen) > 0
    # each phase function, reflectionFed for every particle, and
    # reflectionFed for particles placed to cross the membrane, called
    # directly on the state of step 89
    st = snaps[89]
    for name, call_ref, call_orc in (
            ("collide", lambda: R.call_collide(91), lambda: orc.collide(91)),
            ("llist", R.call_llist, orc.llist_update),
            ("totalva", R.call_totalva, orc.total_va),
            ("pfdt", R.call_pfdt, orc.pfdt),
            ("forces", R.call_forces, orc.forces)):
        R.set_state(st)
        orc.set_state(st)
        call_ref()
        call_orc()
        a, b = R.get_state(89), orc.get_state()
        assert _diff(a, b) == {}, name
        assert a.s["Sarea"] == b.s["Sarea"], name
    R.set_state(st)
    orc.set_state(st)
    fr = np.array([R.call_reflection(i) for i in range(st.ns)])
    fo = np.array([orc.reflection(i) for i in range(st.ns)])
    assert np.array_equal(fr, fo)
    assert _diff(R.get_state(89), orc.get_state()) == {}
    _check_crossings(R, orc, st, M, 200, 89)
