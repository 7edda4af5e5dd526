"""The autotuner's search and cache on the CPU (a host-only plan and a
modelled timer in place of CUDA events): one pass of coordinate descent from
the defaults keeps the fastest setting of each option, applies it to the
plan, and a plan of the same pattern gets the remembered choice without
timing."""
import chompack_b200 as cp
from chompack_b200 import autotune as T
from chompack_b200.plan import Plan
from helpers import problem

COST = {
    "subtrees": {1: 0.0, 0: 1.0},
    "small_front_nj": {64: 0.0, 48: -0.5, 32: -1.0, 0: 2.0},
    "pinv_ksplit": {512: 0.0, 384: 0.3, 768: -0.2, 1024: 0.1},
    "chol_ksplit": {0: 0.0, 256: 1.0, 512: -0.1},
}


def _timer(calls):
    def timer(plan):
        calls.append(1)
        return 10.0 + sum(COST[name][plan.option(name)] for name in COST)
    return timer


def test_coordinate_descent_and_cache():
    T._cache.clear()
    A, s = problem("grid2d", 20, merge=(8, 8), seed=1)
    plan = Plan(s, device=-1)
    calls = []
    rep = T.tune(plan, None, timer=_timer(calls))
    assert rep["cached"] is False
    assert rep["choice"]["subtrees"] == 1 and rep["choice"]["small_front_nj"] == 32
    assert rep["choice"]["pinv_ksplit"] == 768 and rep["choice"]["chol_ksplit"] == 512
    assert abs(rep["ms"] - (10.0 - 1.0 - 0.2 - 0.1)) < 1e-12 and rep["default_ms"] == 10.0
    assert plan.options()["small_front_nj"] == 32 and plan.options()["pinv_ksplit"] == 768
    n_trials = 1 + sum(len(v) - 1 for _, v in T.CANDIDATES)
    assert len(calls) == n_trials == len(rep["trials"])
    # same pattern, new plan: the remembered choice, no timing
    A2, s2 = problem("grid2d", 20, merge=(8, 8), seed=7)      # other values, same pattern
    plan2 = Plan(s2, device=-1)
    calls2 = []
    rep2 = T.tune(plan2, None, timer=_timer(calls2))
    assert rep2["cached"] is True and not calls2
    assert plan2.options() == plan.options()
    # another pattern is timed again
    A3, s3 = problem("grid2d", 21, merge=(8, 8), seed=1)
    calls3 = []
    assert T.tune(Plan(s3, device=-1), None, timer=_timer(calls3))["cached"] is False and calls3
    T._cache.clear()


def test_options_round_trip_and_defaults():
    A, s = problem("grid2d", 12, seed=2)
    plan = Plan(s, device=-1)
    d = plan.options()
    assert d["small_front_nj"] == 64 and d["subtrees"] == 1 and d["pinv_ksplit"] == 512 and d["chol_ksplit"] == 0
    plan.set_option("small_front_nj", 0)
    plan.set_option("chol_ksplit", 300)         # rounded down to a multiple of 64
    assert plan.option("small_front_nj") == 0 and plan.option("chol_ksplit") == 256
    plan.set_option("small_front_nj", None)
    assert plan.option("small_front_nj") == 64
