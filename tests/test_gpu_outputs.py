"""The library's writers and MAIN against the reference's own output files
(tests/golden/outputs, written by the reference's main(): see
make_output_fixtures.py there), byte for byte: irbc_write_rbcdata and
irbc_write_stl from the vertex state the reference's record was written
from, and MAIN's knobs.dat after the same set-up."""
import os
import subprocess
import tempfile

import pytest

import helpers as H
import test_outputs as TO

pytestmark = [pytest.mark.gpu, TO.pytestmark]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAIN = os.path.join(ROOT, "irbc-code_b200", "MAIN")


def test_library_writers_reproduce_the_reference_files():
    import irbc_b200 as G
    fx = TO.fixture_state()
    V, E, T = H.troph()
    sim = G.Simulation(G.default_params(Ns=40000, seed=int(fx["seed"])))
    sim.init(V, E, T, int(fx["knobs"]))
    sim.set_state(TO.with_fixture_vertices(sim.get_state(), fx))
    d = tempfile.mkdtemp(prefix="irbc_gout_")
    sim.write_rbcdata(os.path.join(d, "RBCdata.dat"), append=False)
    sim.write_stl(os.path.join(d, "rbc1.stl"))
    assert open(os.path.join(d, "RBCdata.dat"), "rb").read() == TO.read("RBCdata.dat")
    assert open(os.path.join(d, "rbc1.stl"), "rb").read() == TO.read("rbc1.stl")
    sim.close()


def test_main_writes_the_reference_knobs_file(tmp_path):
    fx = TO.fixture_state()
    env = dict(os.environ, IRBC_STEPS="1", IRBC_NS="40000", IRBC_SEED=str(int(fx["seed"])))
    vf, ef, tf = H.O.troph_files()
    r = subprocess.run([MAIN, "0.005", "0.015", vf, ef, tf, str(int(fx["knobs"])), "RBCdata.dat", "0"],
                       cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "knobs.dat").read_bytes() == TO.read("knobs.dat")
