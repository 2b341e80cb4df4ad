"""The precision study's host-side statistics (no GPU): ensemble means,
their differences and the sampling noise, on synthetic per-seed summaries."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "irbc-code_b200"))


def _summary(profile, shear, temp, area, vol, bonds, com, drift=0.0, roll_var=1e-4):
    return dict(profile=np.asarray(profile, float), shear=shear, temperature=temp, area=area, volume=vol,
                bonds=bonds, com_velocity=com, temperature_drift=drift, area_drift=drift, volume_drift=drift,
                bonds_series=np.full(5, float(bonds)), rolling_mean=com, rolling_var=roll_var)


def test_identical_ensembles_have_zero_error():
    from irbc_b200 import precision
    prof = np.linspace(0.0, 0.1, 38)
    a = [_summary(prof * (1 + 0.01 * k), 0.0025, 1.0 + 0.001 * k, 500.0, 840.0, 10.0 + k, 0.01) for k in range(4)]
    err = precision.compare({"fp64": a, "fp32": [dict(r) for r in a], "wallspeed": 0.1})
    for key in ("profile_l2_rel", "shear_rel", "temperature_rel", "area_rel", "volume_rel", "bonds_abs",
                "com_velocity_abs", "temperature_drift_abs", "area_drift_abs", "volume_drift_abs",
                "bonds_series_max_abs", "rolling_mean_abs", "rolling_var_rel"):
        assert err[key] == 0.0, key
    assert err["seeds"] == 4
    assert err["noise_temperature_rel"] > 0.0


def test_known_offsets_and_noise():
    from irbc_b200 import precision
    prof = np.linspace(0.0, 0.1, 38)
    a = [_summary(prof, 0.0025, 1.0 + d, 500.0, 840.0, 10.0, 0.010) for d in (-0.01, 0.01)]
    b = [_summary(prof * 1.02, 0.0025 * 1.01, 1.0 + d, 505.0, 840.0, 11.0, 0.012, drift=1e-3, roll_var=1.5e-4)
         for d in (-0.01, 0.01)]
    err = precision.compare({"fp64": a, "fp32": b, "wallspeed": 0.1})
    assert err["profile_l2_rel"] == pytest.approx(0.02)
    assert err["shear_rel"] == pytest.approx(0.01)
    assert err["area_rel"] == pytest.approx(0.01)
    assert err["volume_rel"] == 0.0
    assert err["bonds_abs"] == pytest.approx(1.0)
    assert err["com_velocity_abs"] == pytest.approx(0.02)
    assert err["rolling_mean_abs"] == pytest.approx(0.02)
    assert err["area_drift_abs"] == pytest.approx(1e-3)
    assert err["bonds_series_max_abs"] == pytest.approx(1.0)
    assert err["rolling_var_rel"] == pytest.approx(0.5)
    # two seeds of +-0.01 on each side: s.e. of the difference = sqrt(2 * 2e-4 / 2)
    assert err["noise_temperature_rel"] == pytest.approx(np.sqrt(2e-4))


def test_developed_couette_adds_the_linear_profile():
    from irbc_b200 import precision, State
    st = State.__new__(State)
    st.ns, st.nv, st.nlig, st.ncell = 3, 0, 0, 0
    st.a = {"sx": np.zeros(3), "sz": np.array([0.0, 20.0, 40.0]), "svx": np.array([1.0, 1.0, 1.0])}
    st.s = {}
    out = precision.developed_couette(st, 0.1, 40.0)
    assert np.allclose(out.a["svx"], [1.0, 1.05, 1.1])
    assert np.array_equal(st.a["svx"], [1.0, 1.0, 1.0])  # the input is left alone
