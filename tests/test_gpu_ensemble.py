"""Ensemble statistics against the reference itself: the reference's
configuration as shipped (960,000 particles, 60 x 40 x 40, the 600-vertex
mesh with 500 knobs), run for 20,000 steps K times by the reference's own
OpenMP build with its own clock-seeded Mersenne Twister
(tests/golden/ensemble/reference_cfg1.json, written by
oracle/ensemble_study.py), and K times by the FP64 library with seeds
1..K.  Each run gives one window average (steps 10,000-20,000, every 500)
of the solvent temperature of peculiar velocities, the Couette profile,
the bond count, the membrane's rolling velocity, its area and volume.

Bound, per observable: the two ensemble means differ by at most Z
combined standard errors, sqrt(se_gpu^2 + se_ref^2), with Z = 4 (the
runs are few, so the standard errors are themselves uncertain); for the
profile, the same per layer."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "golden", "ensemble", "reference_cfg1.json")
Z = 4.0


@pytest.mark.skipif(not os.path.exists(REF), reason="no reference ensemble")
def test_gpu_ensemble_matches_the_reference_ensemble():
    import oracle.ensemble_study as ES
    ref = json.load(open(REF))
    runs = ES.run_gpu(len(ref["runs"]), ref["steps"], ref["start"], ref["every"])
    gpu = ES.summary(runs)
    rs = ref["summary"]
    report = {}
    for k in ("temperature", "bonds", "rolling", "area", "volume"):
        d = abs(gpu[k]["mean"] - rs[k]["mean"])
        bound = Z * np.hypot(gpu[k]["se"], rs[k]["se"])
        report[k] = (gpu[k]["mean"], rs[k]["mean"], bound)
        assert d <= bound, report
    pg, pr = np.array(gpu["profile"]["mean"]), np.array(rs["profile"]["mean"])
    sb = Z * np.hypot(np.array(gpu["profile"]["se"]), np.array(rs["profile"]["se"]))
    assert (np.abs(pg - pr) <= sb).all(), (pg - pr, sb)
