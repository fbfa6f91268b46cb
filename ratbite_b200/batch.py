"""Batched render jobs on one GPU: many jobs of uneven resolution, sample
count and scene size rendered together (no counterpart in the reference,
which renders one scene interactively).

Every job has its own context (scene, light tree, wavefront buffers) on the
same device. The scheduler spreads the jobs over `streams` CUDA streams
(longest job first onto the least-loaded stream, then shortest first within
each stream, which keeps the median completion time low), and renders each
job in calls of `chunk` samples per pixel through rb_render_graph, so a
job's wave sequence is one graph launch per call after the first. All work
is enqueued up front; a job's completion time is a CUDA event after its last
call, against one start event that every stream waits on.

The autotuner picks the stream count, the samples per call and the paths in
flight per job (the wavefront queue capacity) by timing the schedule on a
small, shortened sample of the jobs.
"""
from __future__ import annotations

import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import assets, lighttree, scenes
from .nrc import RadianceCache
from .rendering_interface import RenderingInterface

SIDES = tuple(128 * k for k in range(1, 9))      # square images 128^2 .. 1024^2


@dataclass
class Job:
    index: int
    seed: int
    side: int           # image is side x side
    spp: int
    triangles: int      # target size of the procedural scene
    form: str           # "plain" or "cached" (radiance cache)

    @property
    def paths(self) -> int:
        return self.side * self.side * self.spp


def draw_jobs(seed: int = 5, n: int = 64, forms=("plain", "cached")) -> list[Job]:
    """n jobs from a seed: side uniform over {128, 256, ..., 1024} (image
    sizes 128^2 .. 1024^2 in steps of 128 per side), spp log-uniform in
    [16, 1024], scene size log-uniform in [10^4, 2 x 10^6] triangles, form
    uniform over `forms`."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        side = int(SIDES[rng.integers(len(SIDES))])
        spp = int(round(math.exp(rng.uniform(math.log(16), math.log(1024)))))
        tris = int(round(math.exp(rng.uniform(math.log(1e4), math.log(2e6)))))
        form = forms[int(rng.integers(len(forms)))]
        jobs.append(Job(i, seed * 1000 + i, side, spp, tris, form))
    return jobs


@dataclass
class Schedule:
    streams: int = 4
    chunk: int = 64                 # samples per pixel per render call
    max_paths: int = 2 << 20        # wavefront capacity per job

    def capacity(self, job: Job) -> int:
        return min(job.side * job.side * min(self.chunk, job.spp), self.max_paths)


@dataclass
class Result:
    schedule: Schedule
    total_paths: int
    seconds: float                  # start to the last job's completion (device events)
    latencies: list = field(default_factory=list)   # per job, seconds from the start

    @property
    def paths_per_s(self) -> float:
        return self.total_paths / self.seconds

    def percentile(self, q: float) -> float:
        return float(np.percentile(np.array(self.latencies), q))


class BatchRenderer:
    """Holds the jobs' scenes on the host; contexts are created per run."""

    def __init__(self, jobs: list[Job], device: int = 0, max_depth: int = 12, threads: int = 8):
        self.jobs = jobs
        self.device = device
        self.cie, self.basis = assets.cie_xyz(), assets.basis_rgb()
        self.luts = assets.generated_luts(samples=1 << 14, device=device)   # regenerated on the GPU

        def build(job):
            sc = scenes.scale_scene(seed=job.seed, target_tris=job.triangles,
                                    n_emitters=int(min(4096, max(16, job.triangles // 500))),
                                    width=job.side, height=job.side, spp=job.spp, max_depth=max_depth)
            return sc, lighttree.build_for_scene(sc)

        with ThreadPoolExecutor(max_workers=threads) as ex:
            self.scenes = list(ex.map(build, jobs))

    def _assign(self, jobs: list[Job], streams: int) -> list[list[Job]]:
        lanes: list[list[Job]] = [[] for _ in range(streams)]
        load = [0] * streams
        for j in sorted(jobs, key=lambda j: -j.paths):
            k = int(np.argmin(load))
            lanes[k].append(j)
            load[k] += j.paths
        for lane in lanes:
            lane.sort(key=lambda j: j.paths)
        return lanes

    def run(self, schedule: Schedule, jobs: list[Job] | None = None, spp_cap: int | None = None,
            keep_images: bool = False) -> Result:
        """Renders `jobs` (default: all) under `schedule`; spp_cap shortens
        every job (autotuning). Contexts are set up, and wave buffers and
        graphs allocated by one untimed call each, before the timed region."""
        import torch

        jobs = list(self.jobs if jobs is None else jobs)
        torch.cuda.set_device(self.device)
        spp_of = {j.index: (min(j.spp, spp_cap) if spp_cap else j.spp) for j in jobs}
        ctxs, caches = {}, {}
        for j in jobs:
            sc, lt = self.scenes[j.index]
            ri = RenderingInterface(device=self.device, max_paths_in_flight=schedule.capacity(j))
            ri.load_scene(sc, self.luts, self.cie, self.basis, light_tree=lt, max_depth=sc.max_depth)
            if j.form == "cached":
                caches[j.index] = RadianceCache(device=self.device, seed=j.seed)
                ri.attach_radiance_cache(caches[j.index])
            ctxs[j.index] = ri
        streams = [torch.cuda.Stream(device=self.device) for _ in range(schedule.streams)]
        lanes = self._assign(jobs, schedule.streams)
        # untimed warm-up: allocate every job's buffers and capture its graph shapes
        for k, lane in enumerate(lanes):
            for j in lane:
                n = spp_of[j.index]
                sizes = {min(schedule.chunk, n)} | ({n % schedule.chunk} if n % schedule.chunk else set())
                for c in sizes:
                    self._call(ctxs[j.index], j, 1 << 24, c, streams[k])
        torch.cuda.synchronize()
        for ri in ctxs.values():                      # launch counters start here
            ri.get_stats()
            ri.cache_stats() if ri._cache is not None else None
        start = torch.cuda.Event(enable_timing=True)
        start.record(torch.cuda.current_stream())
        for s in streams:
            s.wait_event(start)
        ends = {}
        t0 = time.perf_counter()
        for k, lane in enumerate(lanes):
            for j in lane:
                n = spp_of[j.index]
                for off in range(0, n, schedule.chunk):
                    self._call(ctxs[j.index], j, off, min(schedule.chunk, n - off), streams[k])
                e = torch.cuda.Event(enable_timing=True)
                e.record(streams[k])
                ends[j.index] = e
        torch.cuda.synchronize()
        host_s = time.perf_counter() - t0
        lat = [start.elapsed_time(ends[j.index]) / 1e3 for j in jobs]
        images = {j.index: ctxs[j.index].read_accumulation() for j in jobs} if keep_images else None
        launches = 0
        for ri in ctxs.values():
            st = ri.get_stats()
            launches += (st.launches_generate + st.launches_extend + st.launches_shade + st.launches_nee
                         + st.launches_bsdf + st.launches_shadow + st.launches_resolve)
            if ri._cache is not None:
                launches += ri.cache_stats().launches
        for j in jobs:
            assert ctxs[j.index].status().flags == 0
            ctxs[j.index].cleanup()
        for c in caches.values():
            c.close()
        res = Result(schedule, sum(j.side * j.side * spp_of[j.index] for j in jobs), max(lat), lat)
        res.host_seconds = host_s
        res.images = images
        res.gpu_launches = launches
        return res

    @staticmethod
    def _call(ri, job: Job, offset: int, count: int, stream):
        if job.form == "cached":
            ri.render(offset, count, stream=stream.cuda_stream)
        else:
            ri.render_graph(offset, count, stream=stream.cuda_stream)

    def autotune(self, candidates=None, sample: int = 12, spp_cap: int = 32) -> tuple[Schedule, list]:
        """Times each candidate schedule on `sample` jobs (spread over the
        job sizes) shortened to spp_cap samples, and returns the one with the
        highest throughput with the table of trials."""
        if candidates is None:
            candidates = [Schedule(s, c, 2 << 20) for s in (4, 8, 16) for c in (32, 64, 128)]
        order = sorted(self.jobs, key=lambda j: j.paths)
        pick = [order[int(i)] for i in np.linspace(0, len(order) - 1, min(sample, len(order)))]
        trials = []
        for cand in candidates:
            r = self.run(cand, jobs=pick, spp_cap=spp_cap)
            trials.append((cand, r.paths_per_s))
        best = max(trials, key=lambda t: t[1])[0]
        return best, trials
