"""MAIN, the reference's command line over the library: same arguments, the
set-up printout, knobs.dat, RBCdata.dat records and rbc<k>.stl files; its
records equal what the Python binding writes for the same simulation."""
import os
import subprocess

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAIN = os.path.join(ROOT, "irbc-code_b200", "MAIN")
TROPH = [os.path.join(ROOT, "tests", "golden", "troph600", n) for n in ("TrophV600.dat", "TrophE600.dat",
                                                                      "TrophT600.dat")]


def test_main_writes_the_reference_files(tmp_path):
    env = dict(os.environ, IRBC_STEPS="25", IRBC_OUT_EVERY="10")
    r = subprocess.run([MAIN, "0.005", "0.015"] + TROPH + ["500", "RBCdata.dat", "1"], cwd=tmp_path, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    for key in ("Mean edge is:", "Standard deviation is:", "Sarea:", "Volume:", "Shear modulus::",
                "Young's modulus::", "Poisson's ratio::", "no of vertices selected:\t500"):
        assert key in out, key
    knobs = np.loadtxt(tmp_path / "knobs.dat")
    assert knobs.shape == (500, 3)
    text = (tmp_path / "RBCdata.dat").read_text().splitlines()
    heads = [i for i, l in enumerate(text) if l.startswith("#")]
    assert [text[i] for i in heads] == ["#1", "#2"]     # after steps 10 and 20
    assert heads[1] - heads[0] == 601 and len(text) == 2 * 601
    assert (tmp_path / "rbc1.stl").exists() and (tmp_path / "rbc2.stl").exists()
    # the same simulation through the Python binding, first record
    import irbc_b200 as G
    from irbc_b200 import mesh
    p = G.default_params(onrate=0.005, offrate=0.015, Nt=600, out_every=10)
    sim = G.Simulation(p)
    V, E, T = mesh.read_reference_files(*TROPH)
    sim.init(V, E, T, 500)
    sim.step(11)
    ref = tmp_path / "ref.dat"
    sim.write_rbcdata(str(ref), False)
    assert ref.read_text().splitlines() == text[:601]
    sim.close()


def test_record_async_matches_state():
    """irbc_record_async packs x, y, z, ix, iy, bondi of every vertex into a
    page-locked buffer; after sync it equals the state's vertex fields."""
    import numpy as np
    import irbc_b200 as G
    op, orc = H.make_oracle(ns=20000, seed=5, onrate=300.0, offrate=50.0)
    sim = H.gpu_like(op, orc, 5)
    sim.step(7)
    buf = G.PinnedArray(sim.record_bytes(), np.uint8)
    sim.record_async(buf)
    sim.sync()
    st = sim.get_state()
    nv = sim.nv
    a = buf.array
    d = a[:24 * nv].view(np.float64)
    q = a[24 * nv:].view(np.int32)
    for k, name in enumerate(("x", "y", "z")):
        assert np.array_equal(d[k * nv:(k + 1) * nv], st.a[name]), name
    for k, name in enumerate(("ix", "iy", "bondi")):
        assert np.array_equal(q[k * nv:(k + 1) * nv], st.a[name]), name
    sim.close()
