"""The launch-schedule autotuner's host logic, on CPU: irbc_tune_select
driven by a fake timer, and the batch schedule's argument checks (a batch
with no members makes no CUDA call)."""
import ctypes as C

import pytest

import irbc_b200 as G


class FakeTimer:
    """Candidate i takes times[i][k] on its k-th run (the last value
    repeats); None marks a candidate that cannot run."""

    def __init__(self, times):
        self.times = times
        self.calls = [0] * len(times)

    def __call__(self, i):
        k = self.calls[i]
        self.calls[i] += 1
        t = self.times[i]
        if t is None:
            return None
        return t[min(k, len(t) - 1)]


def test_picks_the_fastest_candidate():
    best, med = G.tune_select(3, FakeTimer([[1.0], [0.7], [0.8]]), repeats=3, margin=0.02)
    assert best == 1
    assert med == [1.0, 0.7, 0.8]


def test_incumbent_kept_within_the_margin():
    # 1% faster is not enough to displace candidate 0 at a 2% margin
    assert G.tune_select(2, FakeTimer([[1.0], [0.99]]), margin=0.02)[0] == 0
    assert G.tune_select(2, FakeTimer([[1.0], [0.97]]), margin=0.02)[0] == 1
    # a later candidate has to beat the best so far, not only candidate 0
    assert G.tune_select(3, FakeTimer([[1.0], [0.9], [0.89]]), margin=0.02)[0] == 1


def test_warm_up_run_is_not_scored_and_median_ignores_one_outlier():
    # candidate 1: a slow first run (graph capture, first launches), then
    # 0.5, one 9.0 outlier, 0.5
    ft = FakeTimer([[1.0], [50.0, 0.5, 9.0, 0.5]])
    best, med = G.tune_select(2, ft, repeats=3)
    assert best == 1 and med[1] == 0.5
    assert ft.calls == [4, 4]
    # an even count of timed runs takes the middle pair's mean
    best, med = G.tune_select(1, FakeTimer([[0.0, 1.0, 2.0, 3.0, 4.0]]), repeats=4)
    assert med[0] == 2.5


def test_candidates_that_cannot_run_are_skipped():
    ft = FakeTimer([[1.0], None, [0.5]])
    best, med = G.tune_select(3, ft, repeats=2)
    assert best == 2
    assert med == [1.0, -1.0, 0.5]
    assert ft.calls == [3, 1, 3]
    # an infeasible incumbent: the first feasible candidate takes its place
    best, med = G.tune_select(3, FakeTimer([None, [2.0], [1.99]]), margin=0.02)
    assert best == 1 and med[0] == -1.0


def test_every_candidate_infeasible_is_a_capacity_error():
    L = G.lib()
    fn = G.TUNE_MEASURE(lambda i, ctx, out: G.ERR_CAPACITY)
    best = C.c_int32(7)
    assert L.irbc_tune_select(3, fn, None, 2, 0.0, None, C.byref(best)) == G.ERR_CAPACITY
    assert best.value == 7


def test_other_errors_end_the_search():
    L = G.lib()
    seen = []

    def cb(i, ctx, out):
        seen.append(i)
        if i == 1:
            return -2
        out[0] = 1.0
        return 0

    fn = G.TUNE_MEASURE(cb)
    best = C.c_int32(-1)
    assert L.irbc_tune_select(3, fn, None, 1, 0.0, None, C.byref(best)) == -2
    assert seen == [0, 0, 1]
    # an exception in a Python measure comes back out of tune_select
    def bad(i):
        raise ValueError("boom")
    with pytest.raises(ValueError):
        G.tune_select(2, bad)


def test_argument_checks():
    L = G.lib()
    fn = G.TUNE_MEASURE(lambda i, ctx, out: 0)
    best = C.c_int32(0)
    for n, rep, margin in ((0, 1, 0.0), (2, 0, 0.0), (2, 65, 0.0), (2, 1, 1.0), (2, 1, -0.1)):
        assert L.irbc_tune_select(n, fn, None, rep, margin, None, C.byref(best)) == G.ERR_ARG
    assert L.irbc_tune_select(2, fn, None, 1, 0.0, None, None) == G.ERR_ARG

    # a measurement that is not a time is refused
    def nan(i, ctx, out):
        out[0] = float("nan")
        return 0
    assert L.irbc_tune_select(1, G.TUNE_MEASURE(nan), None, 1, 0.0, None, C.byref(best)) == G.ERR_ARG


def test_batch_schedule_defaults_and_checks():
    b = G.Batch(nthreads=2)
    assert b.schedule() == dict(streams=2, membrane=1, graphs=0, chunk=24, fused=1)
    b.set_schedule(streams=1, graphs=1, chunk=96, fused=0)
    assert b.schedule() == dict(streams=1, membrane=1, graphs=1, chunk=96, fused=0)
    for bad in (dict(streams=3), dict(membrane=0), dict(graphs=2), dict(chunk=30), dict(chunk=0),
                dict(chunk=2424), dict(fused=2)):
        with pytest.raises(G.IrbcError):
            b.set_schedule(**bad)
        assert b.schedule() == dict(streams=1, membrane=1, graphs=1, chunk=96, fused=0)
    L = G.lib()
    s, taken = G.Schedule(), C.c_int64(0)
    # nothing to tune on: no members
    assert L.irbc_batch_autotune(b.b, 24, 1, 0.02, C.byref(s), C.byref(taken)) == -3
    for steps, rep, margin in ((0, 1, 0.0), (24, 0, 0.0), (24, 1, 1.5)):
        assert L.irbc_batch_autotune(b.b, steps, rep, margin, C.byref(s), C.byref(taken)) == G.ERR_ARG
    b.close()
