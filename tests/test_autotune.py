"""Autotuner search logic (host only): coordinate descent finds the minimum of a separable
objective, evaluates each point once, and starts from the defaults."""
import dataclasses

from cfd_b200 import Tuning
from cfd_b200.autotune import CANDIDATES, coordinate_search


def _value(t, knob):
    return tuple(getattr(t, k) for k in knob) if isinstance(knob, tuple) else getattr(t, knob)


def test_coordinate_search_finds_separable_minimum():
    target = {"target_tiles": 148 * 16, "wide_row": 32, "lanes_div": 8, "fuse_first": 1, "sell_rows": 512,
              "krylov_pair": 0, ("tail_rows", "tail_cluster"): (65536, 0)}
    calls = []

    def cost(t):
        calls.append(dataclasses.astuple(t))
        return sum(abs(CANDIDATES[k].index(_value(t, k)) - CANDIDATES[k].index(v)) + 0.5
                   for k, v in target.items())

    best, val, trace = coordinate_search(cost)
    assert all(_value(best, k) == v for k, v in target.items())
    assert val == min(v for _, v in trace)
    assert len(calls) == len(set(calls))          # memoised
    assert trace[0][0] == dataclasses.asdict(Tuning())


def test_coordinate_search_keeps_default_when_flat():
    best, val, trace = coordinate_search(lambda t: 1.0)
    assert best == Tuning() and val == 1.0


def test_retune_knobs_keeps_the_schedule_and_searches_only_its_knobs():
    from cfd_b200.autotune import SCHEDULE_KNOBS, retune_knobs
    base = dataclasses.replace(Tuning(), mixed_sweeps=1, mixed_weight=0.85, wide_row=64)
    seen = []

    def cost(t):
        seen.append(t)
        return 2.0 - (t.tail_rows == 8192)  # the tail pays off only under this schedule

    best, rec = retune_knobs(cost, base)
    assert best.tail_rows == 8192 and rec["ms"] == 1.0 and rec["start_ms"] == 2.0
    assert (best.mixed_sweeps, best.mixed_weight, best.wide_row) == (1, 0.85, 64)
    names = {n for k in SCHEDULE_KNOBS for n in (k if isinstance(k, tuple) else (k,))}
    for t in seen:  # every point differs from the base in the schedule knobs alone
        diff = {k for k, v in dataclasses.asdict(t).items() if v != getattr(base, k)}
        assert diff <= names
