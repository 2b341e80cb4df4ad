"""Output files in the reference's formats, byte for byte (no GPU).

tests/golden/outputs holds what the reference's own main() wrote
(make_output_fixtures.py there): knobs.dat after set-up
(maincode.cpp:435-445), the first RBCdata.dat record, written at the end of
step 5000 (maincode.cpp:746-753), and rbc1.stl beside it (filewrite,
Src/memfuncs.cpp:590-626), with the vertex state that record was written
from.  The oracle's writers must reproduce the two record files from that
state, and its set-up must place the same knobs."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "outputs")
pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(FIX, "state.npz")), reason="no output fixtures")

VERTEX_KEYS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "poff", "pon", "pid", "ix", "iy", "bondi",
               "bondl", "knob")


def fixture_state():
    return np.load(os.path.join(FIX, "state.npz"))


def with_fixture_vertices(st, fx):
    """st (any state of the same simulation) with the fixture's vertex
    state, parasite and counters"""
    out = st.copy()
    for k in VERTEX_KEYS:
        out.a[k][:] = fx[k]
    for k in ("para", "paraV", "paraft", "parafdt"):
        out.s[k] = np.array(fx[k])
    for k, v in zip(("step", "colsteps", "upd", "filecc", "filec"), fx["counters"]):
        out.s[k] = int(v)
    return out


def read(name):
    return open(os.path.join(FIX, name), "rb").read()


def knob_lines(st):
    """knobs.dat as main() writes it: "%lf\\t%lf\\t%lf\\n" per knob vertex"""
    k = st.a["knob"] == 1
    return "".join("%f\t%f\t%f\n" % (x, y, z) for x, y, z in zip(st.a["x"][k], st.a["y"][k], st.a["z"][k])).encode()


def test_oracle_writers_reproduce_the_reference_files():
    fx = fixture_state()
    op = O.default_params(Ns=40000)
    orc = O.Oracle(op, int(fx["seed"]))
    V, E, T = O.load_mesh_files(*O.troph_files())
    orc.init(V, E, T, int(fx["knobs"]))
    assert knob_lines(orc.get_state()) == read("knobs.dat")
    orc.set_state(with_fixture_vertices(orc.get_state(), fx))
    d = tempfile.mkdtemp(prefix="irbc_out_")
    assert orc.write_rbcdata(os.path.join(d, "RBCdata.dat").encode(), 0) == 0
    assert orc.write_stl(os.path.join(d, "rbc1.stl").encode()) == 0
    assert open(os.path.join(d, "RBCdata.dat"), "rb").read() == read("RBCdata.dat")
    assert open(os.path.join(d, "rbc1.stl"), "rb").read() == read("rbc1.stl")
