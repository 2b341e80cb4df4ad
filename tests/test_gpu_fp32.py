"""FP32-bulk solvent against the FP64 oracle.

The solvent is stored and streamed in float, so single-step differences
are bounded by float rounding of positions (~6e-8 relative of the box) and
of the collision's rotation (~1e-7 relative of the velocities).  Cell
indices may differ only for particles within float rounding of a cell face.
The membrane stays FP64."""
import numpy as np
import pytest

import oracle as O
import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def base():
    op, orc = H.make_oracle(ns=40000, seed=41, onrate=300.0, offrate=50.0)
    orc.step(9)
    return op, orc.get_mesh(), orc.get_state()


def _fresh(op, mesh, st, seed=41):
    o = O.Oracle(op, seed)
    o.set_mesh(mesh)
    o.set_state(st)
    return o


def test_fp32_collision_and_stream_steps(base):
    import irbc_b200 as G
    op, mesh, st = base
    o = _fresh(op, mesh, st)
    sim = H.gpu_like(op, o, 41, precision=1, state=st)
    sim.step(2)            # steps 9 and 10 (collision at 10)
    o.step(2)
    g, r = sim.get_state(), o.get_state()
    L = np.array([op.Lx, op.Ly, op.Lz])
    for k, scale in (("sx", op.Lx), ("sy", op.Ly), ("sz", op.Lz)):
        assert np.max(np.abs(g.a[k] - r.a[k])) < 4e-6 * scale, k
    for k in ("svx", "svy", "svz"):
        assert H.rel_err(g.a[k], r.a[k]) < 2e-6, k
    assert (g.a["spid"] != r.a["spid"]).mean() < 1e-3
    assert np.array_equal(g.a["sindio"], r.a["sindio"])
    for k in ("bondi", "bondl", "ix", "iy", "knob"):
        assert np.array_equal(g.a[k], r.a[k]), k
    for k in ("x", "y", "z"):
        assert H.rel_err(g.a[k], r.a[k]) < 1e-9, k


def test_fp32_equals_its_own_restart(base):
    """Exporting and re-importing the FP32 state reproduces the run."""
    import irbc_b200 as G
    op, mesh, st = base
    o = _fresh(op, mesh, st)
    a = H.gpu_like(op, o, 41, precision=1, state=st)
    a.step(5)
    mid = a.get_state()
    b = H.gpu_like(op, o, 41, precision=1, state=mid)
    a.step(15)
    b.step(15)
    assert H.compare(a.get_state(), b.get_state(), 0.0) == {}


def test_fp32_collision_conserves_momentum(base):
    """Away from walls and membrane the SRD rotation conserves each cell's
    momentum; summed over the box the change is the ghost and wall terms
    only, which are zero-mean: check the total is kept to float accuracy."""
    import irbc_b200 as G
    op, mesh, st = base
    o = _fresh(op, mesh, st)
    sim = H.gpu_like(op, o, 41, precision=1, state=st)
    before = sim.get_state()
    sim.call("collide", 10)
    after = sim.get_state()
    bulk = (before.a["sz"] > 2.0) & (before.a["sz"] < op.Lz - 2.0)
    # total kinetic energy stays within the thermostat's bounds
    e0 = np.sum(before.a["svx"] ** 2 + before.a["svy"] ** 2 + before.a["svz"] ** 2)
    e1 = np.sum(after.a["svx"] ** 2 + after.a["svy"] ** 2 + after.a["svz"] ** 2)
    assert abs(e1 - e0) / e0 < 0.05
    assert bulk.sum() > 0.8 * st.ns


def test_fp32_long_run_stays_physical(base):
    """800 steps (list updates and collisions included) in FP32 beside the
    same run in FP64: every particle stays finite and inside the box, and
    the solvent temperature and membrane area agree to a few percent."""
    op, mesh, st = base
    o = _fresh(op, mesh, st)
    f32 = H.gpu_like(op, o, 41, precision=1, state=st)
    f64 = H.gpu_like(op, o, 41, precision=0, state=st)
    f32.step(800)
    f64.step(800)
    g, r = f32.get_state(), f64.get_state()
    for k, L in (("sx", op.Lx), ("sy", op.Ly), ("sz", op.Lz)):
        assert np.isfinite(g.a[k]).all(), k
        assert g.a[k].min() >= -1e-3 and g.a[k].max() <= L + 1e-3, k
    v2g = np.mean(g.a["svx"] ** 2 + g.a["svy"] ** 2 + g.a["svz"] ** 2)
    v2r = np.mean(r.a["svx"] ** 2 + r.a["svy"] ** 2 + r.a["svz"] ** 2)
    assert np.isfinite(v2g) and abs(v2g - v2r) / v2r < 0.05
    assert abs(g.s["Sarea"] - r.s["Sarea"]) / r.s["Sarea"] < 0.02


def test_precision_study_within_one_percent():
    """The precision study on the reference's own configuration (define.h
    box, the shipped mesh, 500 knobs) in developed Couette flow: FP64 and
    FP32-bulk runs for four seeds, 16,000 steps each, sampled every 160.
    Temperature, membrane area and volume and the shear rate of the FP32
    ensemble within 1% of the FP64 ensemble.  The velocity profile and the
    centre-of-mass velocity are sampling-noise limited over this window:
    FP32's difference must be within 1%, or within three standard errors
    of the difference of the ensemble means."""
    import irbc_b200 as G
    from irbc_b200 import precision
    V, E, T = H.troph()
    p = G.default_params(onrate=0.005, offrate=0.015, Nt=600)
    study = precision.run_study(p, V, E, T, 500, 16000, 160, seeds=(71, 72, 73, 74))
    err = precision.compare(study)
    print(err)
    for k, v in err.items():
        assert np.isfinite(v), k
    assert err["temperature_rel"] < 0.01
    assert err["area_rel"] < 0.01 and err["volume_rel"] < 0.01
    assert err["shear_rel"] < max(0.01, 3.0 * err["noise_shear_rel"])
    assert err["profile_l2_rel"] < max(0.01, 3.0 * err["noise_profile_l2_rel"])
    assert err["com_velocity_abs"] < max(0.01, 3.0 * err["noise_com_velocity_abs"])

