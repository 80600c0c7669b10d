"""Autotuner search logic (host only): coordinate descent finds the minimum of a separable
objective, evaluates each point once, and starts from the defaults."""
import dataclasses

from cfd_b200 import Tuning
from cfd_b200.autotune import CANDIDATES, coordinate_search


def test_coordinate_search_finds_separable_minimum():
    target = {"target_tiles": 148 * 16, "wide_row": 32, "lanes_div": 8, "fuse_first": 1, "sell_rows": 512,
              "krylov_pair": 0, "tail_rows": 8192}
    calls = []

    def cost(t):
        calls.append(dataclasses.astuple(t))
        return sum(abs(CANDIDATES[k].index(getattr(t, k)) - CANDIDATES[k].index(v)) + 0.5
                   for k, v in target.items())

    best, val, trace = coordinate_search(cost)
    assert {k: v for k, v in dataclasses.asdict(best).items() if k in target} == target
    assert val == min(v for _, v in trace)
    assert len(calls) == len(set(calls))          # memoised
    assert trace[0][0] == dataclasses.asdict(Tuning())


def test_coordinate_search_keeps_default_when_flat():
    best, val, trace = coordinate_search(lambda t: 1.0)
    assert best == Tuning() and val == 1.0
