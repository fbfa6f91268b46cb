"""Batched render jobs on one GPU: many jobs of uneven resolution, sample
count and scene size rendered together (no counterpart in the reference,
which renders one scene interactively).

Every job has its own context (scene, light tree, accumulation) on the same
device. The plain jobs render in one shared wavefront (rb_render_jobs):
waves are filled with whole sample planes of the jobs, shortest job first
(which keeps the median completion time low), and every kernel of a wave
serves all of its jobs' paths. Jobs of the cached form (the radiance cache,
whose network is per job) render on their own contexts on `streams` CUDA
streams alongside, in calls of `chunk` samples per pixel. A job's
completion time is a CUDA event recorded after the wave (or call) that
finishes it, against one start event.

The autotuner picks the shared wavefront's queue capacity (paths in flight
per wave) and its grid size (blocks launched per kernel, as a percentage of
the resident maximum), and the stream count of the cached jobs, by timing
the schedule on a small, shortened sample of the jobs.
"""
from __future__ import annotations

import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import assets, lighttree, scenes
from .nrc import RadianceCache
from .rendering_interface import RenderingInterface, render_jobs

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
    max_paths: int = 8 << 20        # shared wavefront: paths in flight per wave (queue capacity)
    grid_percent: int = 100         # shared wavefront: blocks per kernel launch, % of the resident maximum
    streams: int = 4                # cached jobs: CUDA streams
    chunk: int = 64                 # cached jobs: samples per pixel per render call

    def capacity(self, job: Job) -> int:
        """Wavefront capacity of a cached job's own context."""
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
    """Holds the jobs' scenes on the host; contexts are created per run.
    tables: (cie_xyz, basis_rgb, luts) for every job (default: the built-in
    stand-ins with LUTs regenerated on the GPU)."""

    def __init__(self, jobs: list[Job], device: int = 0, max_depth: int = 12, threads: int = 8, tables=None):
        self.jobs = jobs
        self.device = device
        if tables is None:
            tables = (assets.cie_xyz(), assets.basis_rgb(), assets.generated_luts(samples=1 << 14, device=device))
        self.cie, self.basis, self.luts = tables

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
        every job (autotuning). Contexts are set up, and wave buffers
        allocated by one untimed call each, before the timed region."""
        import torch

        jobs = list(self.jobs if jobs is None else jobs)
        torch.cuda.set_device(self.device)
        spp_of = {j.index: (min(j.spp, spp_cap) if spp_cap else j.spp) for j in jobs}
        plain = sorted([j for j in jobs if j.form == "plain"], key=lambda j: (j.side * j.side * spp_of[j.index], j.index))
        cached = [j for j in jobs if j.form != "plain"]
        ctxs, caches = {}, {}
        for j in jobs:
            sc, lt = self.scenes[j.index]
            cap = schedule.max_paths if j.form == "plain" else schedule.capacity(j)
            ri = RenderingInterface(device=self.device, max_paths_in_flight=cap)
            ri.load_scene(sc, self.luts, self.cie, self.basis, light_tree=lt, max_depth=sc.max_depth)
            if j.form == "cached":
                caches[j.index] = RadianceCache(device=self.device, seed=j.seed)
                ri.attach_radiance_cache(caches[j.index])
            ctxs[j.index] = ri
        streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, schedule.streams))]
        shared = torch.cuda.Stream(device=self.device)
        lanes = self._assign(cached, len(streams))
        plain_ris = [ctxs[j.index] for j in plain]

        def shared_call(offsets, counts, events=None):
            render_jobs(plain_ris, offsets, counts, max_paths=schedule.max_paths, grid_percent=schedule.grid_percent,
                        done_events=events, stream=shared.cuda_stream)

        # untimed warm-up: the shared wave's buffers, every cached job's buffers
        if plain:
            shared_call([1 << 24] * len(plain), [1] * len(plain))
        for k, lane in enumerate(lanes):
            for j in lane:
                ctxs[j.index].render(1 << 24, min(schedule.chunk, spp_of[j.index]), stream=streams[k].cuda_stream)
        torch.cuda.synchronize()
        for ri in ctxs.values():                      # launch counters start here
            ri.get_stats()
            ri.cache_stats() if ri._cache is not None else None
        ends = {j.index: torch.cuda.Event(enable_timing=True) for j in jobs}
        for e in ends.values():
            e.record()                               # creates the events (the shared call records them again)
        start = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(torch.cuda.current_stream())
        for s in streams + [shared]:
            s.wait_event(start)
        t0 = time.perf_counter()
        for k, lane in enumerate(lanes):
            for j in lane:
                n = spp_of[j.index]
                for off in range(0, n, schedule.chunk):
                    ctxs[j.index].render(off, min(schedule.chunk, n - off), stream=streams[k].cuda_stream)
                ends[j.index].record(streams[k])
        if plain:
            shared_call([0] * len(plain), [spp_of[j.index] for j in plain], [ends[j.index] for j in plain])
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

    def autotune(self, candidates=None, sample: int = 8, spp_cap: int = 16) -> tuple[Schedule, list]:
        """Times each candidate schedule on `sample` jobs (spread over the
        job sizes) shortened to spp_cap samples, and returns the one with the
        highest throughput with the table of trials."""
        if candidates is None:
            candidates = [Schedule(m << 20, g, 4, 64) for m in (4, 16) for g in (50, 100, 200)]
        order = sorted(self.jobs, key=lambda j: j.paths)
        pick = [order[int(i)] for i in np.linspace(0, len(order) - 1, min(sample, len(order)))]
        trials = []
        for cand in candidates:
            r = self.run(cand, jobs=pick, spp_cap=spp_cap)
            trials.append((cand, r.paths_per_s))
        best = max(trials, key=lambda t: t[1])[0]
        return best, trials
