"""Host logic of the batched-jobs scheduler (ratbite_b200.batch), no GPU:
the job draw (ranges, determinism, log-uniform spread), the wavefront
capacity of a schedule, and the longest-first assignment of jobs to streams.
"""
from __future__ import annotations

import math

import numpy as np

from ratbite_b200 import batch


def test_job_draw_is_deterministic_and_in_range():
    a, b = batch.draw_jobs(seed=5, n=64), batch.draw_jobs(seed=5, n=64)
    assert a == b
    assert batch.draw_jobs(seed=6, n=64) != a
    for j in a:
        assert j.side in batch.SIDES
        assert 16 <= j.spp <= 1024
        assert 10_000 <= j.triangles <= 2_000_000
        assert j.form in ("plain", "cached")
    # log-uniform: the median of log(spp) is near the middle of [log 16, log 1024]
    med = np.median([math.log(j.spp) for j in batch.draw_jobs(seed=1, n=2000)])
    assert abs(med - 0.5 * (math.log(16) + math.log(1024))) < 0.15
    assert {j.form for j in a} == {"plain", "cached"}


def test_schedule_capacity():
    s = batch.Schedule(max_paths=1 << 20, grid_percent=100, streams=4, chunk=64)
    small = batch.Job(0, 0, 128, 16, 10_000, "plain")
    big = batch.Job(1, 0, 1024, 512, 10_000, "plain")
    assert s.capacity(small) == 128 * 128 * 16
    assert s.capacity(big) == 1 << 20


def test_assignment_balances_streams():
    jobs = batch.draw_jobs(seed=5, n=64)
    lanes = batch.BatchRenderer._assign(None, jobs, 4)
    assert sorted(j.index for lane in lanes for j in lane) == list(range(64))
    loads = [sum(j.paths for j in lane) for lane in lanes]
    # longest-processing-time assignment: no stream exceeds the mean by more than the largest job
    assert max(loads) - sum(loads) / 4 <= max(j.paths for j in jobs)
    for lane in lanes:
        assert [j.paths for j in lane] == sorted(j.paths for j in lane)
