#!/usr/bin/env python3
"""Generates the output-format fixtures of tests/golden/outputs from the
reference itself (run here, where the reference build oracle/_ref/small
exists; the fixtures then travel without it).

The reference's own main() (replay build: its Mersenne Twister replaced by
the shared counter draw stream, seed 2024) runs the shipped 600-vertex mesh
with 500 knobs and stl_flag 1 until its first RBCdata record, written at
the end of step 5000 (maincode.cpp:746-760).  Kept from its working folder:

  knobs.dat     the knob positions after placement (maincode.cpp:435-445)
  RBCdata.dat   record #1: vertex x y z ix iy bondi (%lf / %d)
  rbc1.stl      filewrite's STL text (Src/memfuncs.cpp:590-626)

The oracle, which equals the reference bit for bit, is stepped to the end
of the same step 5000, and the vertex state the record was written from is
kept as state.npz.  Before anything is written, the oracle's own writers
must reproduce the reference's RBCdata.dat and rbc1.stl byte for byte from
that state: that is what pins the state to the files.
"""
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

SEED, KNOBS, RECORD_STEP = 2024, 500, 5000
VERTEX_KEYS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "poff", "pon", "pid", "ix", "iy", "bondi",
               "bondl", "knob")


def main():
    import oracle as O
    # one thread: the reference's force sums follow its OpenMP schedule, and
    # only the one-thread order is the oracle's (bit for bit)
    R = O.Reference("small", threads=1)
    vf, ef, tf = O.troph_files()
    wd = tempfile.mkdtemp(prefix="irbc_outfix_")
    # stop at step RECORD_STEP + 1's TotalVA: the record of step RECORD_STEP is written
    assert R.run(vf, ef, tf, KNOBS, RECORD_STEP + 1, seed=SEED, workdir=wd, stl=1) == 0
    for name in ("knobs.dat", "RBCdata.dat", "rbc1.stl"):
        assert os.path.exists(os.path.join(wd, name)), name
    orc = O.Oracle(R.p, SEED)
    V, E, T = O.load_mesh_files(vf, ef, tf)
    orc.init(V, E, T, KNOBS)
    orc.step(RECORD_STEP + 1)  # steps 0 .. RECORD_STEP
    st = orc.get_state()
    assert st.s["filec"] == 1, st.s["filec"]
    check = tempfile.mkdtemp(prefix="irbc_outchk_")
    assert orc.write_rbcdata(os.path.join(check, "RBCdata.dat").encode(), 0) == 0
    assert orc.write_stl(os.path.join(check, "rbc1.stl").encode()) == 0
    for name in ("RBCdata.dat", "rbc1.stl"):
        a = open(os.path.join(wd, name), "rb").read()
        b = open(os.path.join(check, name), "rb").read()
        if a != b:
            la, lb = a.decode().splitlines(), b.decode().splitlines()
            bad = [(i, x, y) for i, (x, y) in enumerate(zip(la, lb)) if x != y]
            raise SystemExit("%s: the oracle's writer differs from the reference's in %d of %d lines, first %s"
                             % (name, len(bad), len(la), bad[:3]))
    for name in ("knobs.dat", "RBCdata.dat", "rbc1.stl"):
        shutil.copy(os.path.join(wd, name), os.path.join(HERE, name))
    np.savez_compressed(os.path.join(HERE, "state.npz"),
                        **{k: st.a[k] for k in VERTEX_KEYS},
                        para=st.s["para"], paraV=st.s["paraV"], paraft=st.s["paraft"], parafdt=st.s["parafdt"],
                        counters=np.array([st.s[k] for k in ("step", "colsteps", "upd", "filecc", "filec")]),
                        seed=SEED, knobs=KNOBS)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
