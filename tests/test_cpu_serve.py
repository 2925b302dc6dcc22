"""Serving-loop host logic without a GPU: admission accounting, the arrival
schedule, percentiles and the memory estimates."""
import math

import torch

from lig_b200.serve import (GaussianSet, MemoryBudget, fit_bytes, percentile, poisson_requests,
                            render_bytes)


def _sets(k=4):
    out = {}
    for i in range(k):
        n = 1000 * (i + 1)
        out[f"s{i}"] = GaussianSet(torch.zeros(n, 2), torch.zeros(n, 3), torch.zeros(n, 3),
                                   512, 512)
    return out


def test_budget_reserve_release_and_refusal():
    b = MemoryBudget(100)
    assert b.try_reserve(60) and not b.try_reserve(50) and b.try_reserve(40)
    assert b.used == 100 and b.peak == 100
    b.release(60)
    assert b.try_reserve(50) and b.used == 90


def test_schedule_is_seeded_poisson_with_the_mix():
    sets = _sets()
    a = poisson_requests(20.0, 200.0, 0.3, sets, seed=5000)
    b = poisson_requests(20.0, 200.0, 0.3, sets, seed=5000)
    assert a == b
    n = len(a)
    assert abs(n - 4000) < 4 * math.sqrt(4000)          # Poisson count
    fits = sum(1 for _, k, _ in a if k == "fit")
    assert abs(fits / n - 0.3) < 0.03
    ts = [t for t, _, _ in a]
    assert ts == sorted(ts) and ts[-1] < 20.0
    for _, k, p in a:
        if k == "fit":
            assert 512 <= p["side"] <= 4096 and p["n"] == min(round(0.2 * p["side"] ** 2), 10**6)
        else:
            assert 256 <= p["side"] <= 4096 and 0.25 <= p["scale"] <= 2.0
            gs = sets[p["set"]]
            assert 0 <= p["origin"][0] <= max(0.0, gs.W - p["side"] / p["scale"])


def test_percentile_and_estimates():
    xs = list(range(1, 101))
    assert percentile(xs, 50) == 50 and percentile(xs, 99) == 99 and percentile(xs, 100) == 100
    assert math.isnan(percentile([], 50))
    gs = _sets(1)["s0"]
    assert render_bytes(gs, 2048, 2048) > render_bytes(gs, 256, 256) > gs.nbytes
    assert fit_bytes(4096, 4096, 10**6) > fit_bytes(512, 512, 50_000) > 0
