"""CPU: bench.py's host-side choices. The encoder headline is the fastest
pruning policy within the 1% cost bound (the cheapest when none is), and
the CPU sample spreads its pictures over the whole batch (all QPs)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _p(speedup, cost):
    return {"speedup": speedup, "cost_increase_pct": cost}


def test_headline_is_the_fastest_policy_within_the_bound():
    pols = [_p(4.0, 3.0), _p(1.2, 0.9), _p(1.5, 1.0), _p(5.4, 7.2), _p(1.1, 0.4)]
    assert bench.pick_headline(pols) is pols[2]


def test_headline_without_a_policy_within_the_bound_is_the_cheapest():
    pols = [_p(4.0, 3.0), _p(2.0, 1.5), _p(5.4, 7.2)]
    assert bench.pick_headline(pols) is pols[1]


def test_cpu_sample_spreads_over_the_batch():
    idx = bench.sample_indices(128, 64)
    assert len(idx) == 64 and len(set(idx)) == 64
    assert {i // 32 for i in idx} == {0, 1, 2, 3}  # every QP group of 32 pictures
    assert bench.sample_indices(4, 16) == [0, 1, 2, 3]
