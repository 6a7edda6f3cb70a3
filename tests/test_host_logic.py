"""Host-side choices that need no GPU: which sort a configuration selects and
how the benchmark names its metric."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sort_mode_follows_the_key_mode():
    from cnb.core.state import sort_mode_for
    from cnb.utils import config as cfgmod
    # auto: the near-sorted path for 63-bit keys, whose order survives a step;
    # the full radix sort for the reference's 30-bit keys, whose low bits do not
    assert sort_mode_for(cfgmod.make(SORT_MODE="auto"), "morton63") == "adaptive"
    assert sort_mode_for(cfgmod.make(SORT_MODE="auto"), "compat30") == "full"
    assert sort_mode_for(cfgmod.make(), "morton63") == "adaptive"   # the default is auto
    for mode in ("full", "adaptive"):
        for keys in ("morton63", "compat30"):
            assert sort_mode_for(cfgmod.make(SORT_MODE=mode), keys) == mode
    with pytest.raises(ValueError):
        sort_mode_for(cfgmod.make(SORT_MODE="fast"), "morton63")


def test_sort_mode_codes_match_the_header():
    from cnb import _lib
    from cnb.core.state import SORT_MODES
    hdr = open(os.path.join(ROOT, "include", "cnb.h")).read()
    assert f"#define CNB_SORT_FULL {SORT_MODES['full']}" in hdr
    assert f"#define CNB_SORT_ADAPTIVE {SORT_MODES['adaptive']}" in hdr
    assert f"#define CNB_SORT_NEAR_CAP {_lib.SORT_NEAR_CAP}" in hdr


def test_bench_metric_names_the_grid_size():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        spec.loader.exec_module(bench)
    finally:
        sys.argv = argv
    assert bench.metric_for(128) == bench.METRIC          # the default run's metric is unchanged
    assert "N=256^3" in bench.metric_for(256) and "128" not in bench.metric_for(256)


def test_lagrangian_allocation_meets_the_global_budget():
    """cnb.controller.allocate: per-bucket angles that minimise the cost while
    at most `allowed` bodies exceed the budget; on a small case the result
    is feasible, no dearer than one fixed angle with the same violations,
    and equal to the exhaustive optimum."""
    import itertools

    import numpy as np

    from cnb.controller import allocate
    rng = np.random.default_rng(5)
    T, G, per = 4, 6, 5
    owner = np.repeat(np.arange(G), per)
    # cost falls and error grows with the angle index; buckets differ in sensitivity
    sens = rng.uniform(0.5, 2.0, G)
    errors = np.stack([np.repeat(sens, per) * (k + 1) * rng.uniform(0.8, 1.2, G * per) for k in range(T)])
    costs = np.stack([np.full(G, 100.0 / (k + 1)) * rng.uniform(0.9, 1.1, G) for k in range(T)])
    budget = float(np.percentile(errors[1], 80))
    allowed = int((errors[1] > budget).sum())
    idx, total, v = allocate(errors, costs, owner, budget, allowed)
    assert v <= allowed
    assert total <= costs[1].sum() + 1e-9
    best = np.inf
    best_at_v = np.inf     # the cheapest allocation with no more violations than the one returned
    for choice in itertools.product(range(T), repeat=G):
        c = np.array(choice)
        viol = sum(int((errors[c[g], owner == g] > budget).sum()) for g in range(G))
        cost = costs[c, np.arange(G)].sum()
        if viol <= allowed:
            best = min(best, cost)
        if viol <= v:
            best_at_v = min(best_at_v, cost)
    assert total <= best * 1.15       # the Lagrangian point is close to the exhaustive optimum
    # and it is exactly the cheapest allocation with at most its own violations
    assert abs(total - best_at_v) <= 1e-9 * best_at_v
