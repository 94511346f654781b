"""Host-side serving policy (no GPU): the request stream and the admission /
round-planning scheduler of continuous batching."""
import math

import numpy as np

from licom4py_gpu_b200.serving import Request, Scheduler, latency_stats, poisson_mix


def test_poisson_mix_statistics():
    reqs = poisson_mix(count=20000, rate=200.0, seed=3)
    arr = np.array([r.arrival for r in reqs])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert abs(np.mean(np.diff(arr)) - 1 / 200.0) < 0.05 / 200.0
    ns = np.array([r.n for r in reqs])
    for n, p in {48: 0.4, 96: 0.35, 192: 0.2, 384: 0.05}.items():
        assert abs(np.mean(ns == n) - p) < 0.015
    steps = np.array([r.nsub for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 5000
    # log-uniform: the median of log(steps) sits mid-way
    assert abs(np.median(np.log(steps)) - 0.5 * (math.log(100) + math.log(5000))) < 0.05
    assert len({r.seed for r in reqs}) == len(reqs)
    assert poisson_mix(count=50, seed=3)[7].seed == reqs[7].seed  # prefix-stable


def test_scheduler_admits_in_order_within_budget():
    size = {12: 10, 24: 40}
    s = Scheduler(budget=60, member_bytes=lambda n: size[n], max_members=3, round_substeps=5)
    reqs = [Request(rid=k, n=n, nsub=ns, seed=k) for k, (n, ns) in enumerate([(12, 7), (24, 3), (24, 12), (12, 2)])]
    for r in reqs:
        s.arrive(r)
    assert [r.rid for r in s.admit()] == [0, 1]     # 10 + 40; the next 24 would exceed 60
    assert s.used == 50
    plan = s.plan_round()
    assert plan == {0: 5, 1: 3}
    done = s.finish_round(plan)
    assert [r.rid for r in done] == [1] and s.used == 10
    assert [r.rid for r in s.admit()] == [2, 3]     # FIFO: the large one first, then the small one
    assert s.used == 60 and len(s.active) == 3
    plan = s.plan_round()
    assert plan == {0: 2, 2: 5, 3: 2}
    assert sorted(r.rid for r in s.finish_round(plan)) == [0, 3]
    plan = s.plan_round()
    assert plan == {2: 5}
    s.finish_round(plan)
    assert s.finish_round(s.plan_round())[0].rid == 2
    assert s.idle and s.used == 0


def test_scheduler_rejects_requests_larger_than_budget_and_caps_members():
    s = Scheduler(budget=100, member_bytes=lambda n: n, max_members=2, round_substeps=10)
    s.arrive(Request(rid=0, n=500, nsub=10, seed=0))
    assert [r.rid for r in s.rejected] == [0]
    for k in range(1, 4):
        s.arrive(Request(rid=k, n=10, nsub=10, seed=k))
    assert len(s.admit()) == 2 and len(s.waiting) == 1


def test_latency_stats():
    reqs = [Request(rid=k, n=12, nsub=1, seed=k, arrival=0.0) for k in range(100)]
    for k, r in enumerate(reqs):
        r.t_done = (k + 1) / 100.0
    st = latency_stats(reqs)
    assert abs(st["p50_s"] - 0.505) < 1e-9 and abs(st["p99_s"] - 0.9901) < 1e-9


def test_scheduler_shortest_first_order():
    s = Scheduler(budget=100, member_bytes=lambda n: 10, max_members=2, round_substeps=10, order="shortest")
    work = [(48, 900), (12, 50), (24, 30), (12, 10)]
    for k, (n, ns) in enumerate(work):
        s.arrive(Request(rid=k, n=n, nsub=ns, seed=k, arrival=0.1 * k))
    assert s.queued == 4
    assert [r.rid for r in s.admit()] == [3, 1]      # 6*12^2*10, then 6*12^2*50 cell-updates
    s.finish_round(s.plan_round())                    # rid 3 done
    assert [r.rid for r in s.admit()] == [2]
    assert s.queued == 1


def test_scheduler_rejects_unknown_order():
    import pytest
    with pytest.raises(ValueError):
        Scheduler(budget=1, member_bytes=lambda n: 1, order="lifo")
