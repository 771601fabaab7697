"""The autotuner's search (seevr_b200.tune.search) with synthetic costs: no
GPU needed."""
from seevr_b200.tune import search


def test_coordinate_descent_finds_separable_minimum():
    cost = lambda s: (s["a"] - 3) ** 2 + abs(s["b"] - 64) + 1.0
    best, trials = search({"a": [1, 2, 3, 4], "b": [32, 64, 128]}, {"a": 1, "b": 32}, cost)
    assert best == {"a": 3, "b": 64}
    assert len({tuple(sorted(s.items())) for s, _ in trials}) == len(trials)  # each timed once


def test_current_setting_wins_ties():
    best, trials = search({"a": [1, 2, 3]}, {"a": 2}, lambda s: 5.0)
    assert best == {"a": 2}
    assert [s["a"] for s, _ in trials] == [2, 1, 3]


def test_second_pass_follows_interaction():
    # the best b depends on a: one pass stops short, two passes reach the optimum
    cost = lambda s: {(1, 1): 5, (1, 2): 6, (2, 1): 4, (2, 2): 1}[(s["a"], s["b"])]
    cands = {"b": [1, 2], "a": [1, 2]}
    one, _ = search(cands, {"a": 1, "b": 1}, cost, passes=1)
    two, _ = search(cands, {"a": 1, "b": 1}, cost, passes=2)
    assert one == {"a": 2, "b": 1} and two == {"a": 2, "b": 2}
