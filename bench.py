"""Benchmark of the per-sample rendering path on B200.

Default workload (the plain method at scale): seeded scene of ~2.03M
triangles from 128 instances of noise-displaced spheres, tori and boxes,
256 materials, 4,096 emissive triangles with lognormal(0, 1.5) radiance in a
Gaussian light tree, a 1024x512 sky + sun environment map whose 2D CDF is
rebuilt every frame; 1920x1080, 256 samples per pixel, depth 12. One step =
one frame: CDF rebuild + 530,841,600 paths. Metric: paths per second.
`--workload cornell` selects the small configuration (Cornell box, 256x256,
64 spp, depth 8).

On one GPU the line also carries `time_to_rmse`: the radiance-cached form
against the plain tracer on the Cornell box at 1920x1080, depth 12 -- device
seconds until each reaches the plain tracer's 1024-spp RMSE against a
4096-spp FP64-accumulated plain render (time_to_rmse() below; --no-ttr skips
it).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       renders through the C ABI (libratbite_b200.so). `value` is device
           time (CUDA events on the render stream, max over ranks); `e2e` is
           the same metric through the public API with the launch parameters
           uploaded and the FP64 accumulation buffer read back to host memory
           inside the timed region, every step.
reference  the reference's own per-sample code compiled host-side
           (oracle/_ref) rendering the same scene on all host cores; each step
           is a bounded sample (a band of rows at a few samples per pixel).

With N GPUs (torchrun) each rank renders its own sample range of the frame
(weak scaling; disjoint Sobol indices) and the FP64 images are summed by one
NCCL all-reduce per step, the combine step of progressive rendering.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# The headline: paths/s of the plain tracer (`value`), and the cached form's
# time to the plain tracer's 1024-spp RMSE against the FP64 oracle
# (`time_to_rmse`, one B200).
METRIC = "paths/s and time-to-RMSE vs FP64 oracle: guided/cached vs plain, 1 B200"

WORKLOADS = {
    "scale": dict(name="scale_2M_tris_1920x1080_256spp_depth12_envcdf_per_frame", width=1920, height=1080,
                  spp=256, depth=12),
    "cornell": dict(name="cornell_box_256x256_64spp_depth8", width=256, height=256, spp=64, depth=8),
    # throughput of the radiance-cached form (queries, training paths and optimiser steps inside the
    # timed frames; the cache keeps training from frame to frame)
    "cached": dict(name="cornell_box_1920x1080_64spp_depth12_radiance_cache", width=1920, height=1080, spp=64,
                   depth=12, cached=True),
}

# Algorithmic HBM bytes per work unit of each wavefront kernel: the path
# state it must stream in and out, plus the per-unit gathers from tables
# larger than L2. Tables that stay cache-resident (materials, LUTs, spectra,
# light-tree nodes, emitter records, the env-map CDF) are not counted.
#   extend  per ray: 32 B ray in + 32 B hit out, plus 80 B per 8-wide node
#           and 48 B per triangle visited (counted by the traversal counters)
#   shadow  per ray: queue 4, shadow o/d 32, L read+write 32 when unoccluded
#           (counted as always), pending contribution 16, plus visits as extend
#   surface per path entering the bounce: queue 4, ray o/d 32, normal 16,
#           flags 8, hit 16 read; the hit triangle 48 + 8; vertex indices 12
#           and three 16-B attribute reads 48; surface record 80 + normal 16 +
#           flags 8 + queue 4 written (for surface records)
#   nee     per surface record: queue 4, record 48, normal 16, flags 8,
#           wavelengths 16 read; record word 16 and the light sample 48 written
#   bsdf    per surface record (both BxDF kernels): queue 4, record 80, ray
#           o/d 32, normal 16, flags 8, wavelengths + pdfs + throughput 48,
#           light sample 32 read; throughput, flags, ray o/d 56, contribution
#           16 and two queue slots 8 written
EXTEND_BYTES_PER_RAY = 32 + 32
SHADOW_BYTES_PER_RAY = 4 + 32 + 32 + 16
SURFACE_BYTES_PER_PATH = 4 + 32 + 16 + 8 + 16 + 56
SURFACE_BYTES_PER_RECORD = 12 + 48 + 80 + 16 + 8 + 4
NEE_BYTES_PER_RECORD = 4 + 48 + 16 + 8 + 16 + 16 + 48
BSDF_BYTES_PER_RECORD = 4 + 80 + 32 + 16 + 8 + 48 + 32 + 56 + 16 + 8
NODE_BYTES, TRI_BYTES = 80, 48


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def bench_tables():
    """CIE curves, RGB basis and multiple-scattering LUTs that both arms
    render with: the reference's own (its bin/*.bin LUT files, and its
    spectral tables from src/core/spectral.cpp, written as data by the oracle
    build into oracle/_ref/bin/spectra.npz), read as plain files so that no
    library is loaded for them. Without the oracle build, the built-in
    stand-ins of ratbite_b200.assets."""
    d = ROOT / "oracle" / "_ref" / "bin"
    names = dict(conductor="albedoConductorLUT.bin", dielectric_outer="albedoDielectricOuterLUT.bin",
                 dielectric_inner="albedoDielectricInnerLUT.bin",
                 reflective_outer="albedoDielectricReflectiveOuterLUT.bin",
                 reflective_inner="albedoDielectricReflectiveInnerLUT.bin", sheen="sheenLUT.bin")
    if (d / "spectra.npz").exists() and all((d / f).exists() for f in names.values()):
        sp = np.load(d / "spectra.npz")
        luts = {k: np.fromfile(d / f, dtype=np.float32) for k, f in names.items()}
        return sp["cie_xyz"], sp["basis_rgb"], luts, "reference (bin/*.bin LUTs, src/core/spectral.cpp curves)"
    from ratbite_b200 import assets
    return assets.cie_xyz(), assets.basis_rgb(), assets.luts(), "built-in stand-ins (ratbite_b200.assets)"


def make_scene(wl: dict):
    from ratbite_b200 import scenes
    cie, basis, luts, tables = bench_tables()
    if wl["name"].startswith("cornell"):
        scene = scenes.cornell_box(seed=1, cie_xyz=cie, width=wl["width"], height=wl["height"], spp=wl["spp"],
                                   max_depth=wl["depth"])
    else:
        scene = scenes.scale_scene(seed=3, width=wl["width"], height=wl["height"], spp=wl["spp"],
                                   max_depth=wl["depth"])
    return scene, cie, basis, luts, tables


def workload_config(scene, wl: dict, world: int, tables: str) -> dict:
    """The `config` object of both arms' lines (identical for the same
    workload)."""
    has_env = getattr(scene, "envmap", None) is not None
    return {"workload": wl["name"], "width": wl["width"], "height": wl["height"], "spp": wl["spp"],
            "max_depth": wl["depth"], "triangles": scene.triangle_count(),
            "emitters": int(sum(len(e["prim"]) for e in scene.emissive)), "materials": len(scene.materials),
            "envmap": list(scene.envmap.shape[1::-1]) if has_env else None,
            "paths_per_step": wl["width"] * wl["height"] * wl["spp"] * world,
            "parallelism": f"sample-range x{world}", "tables": tables,
            "acceleration": wl.get("acceleration", "flat"),
            "l2": "inputs larger than L2 (wavefront path state 388 B per path in flight, "
                  "~6.5 GB at the default 16M paths per wave)"}


# ------------------------------------------------------------- CPU baseline
def _ref_setup(scene, cie, basis, luts):
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import RefLib, load_scene_into_ref
    ref = RefLib()
    keep = load_scene_into_ref(ref, scene, luts, cie, basis)
    return ref, keep


def _strided_sample(ref, wl, cores, target_s):
    """A bounded CPU sample of the frame with the frame's cost mix: every
    stride-th row from top to bottom (all columns), at spp samples per pixel
    (sample indices 0..spp-1), sized to take about target_s on `cores`
    threads. Returns (first_row, stride, spp)."""
    W, H = wl["width"], wl["height"]
    probe_stride = max(1, H // 16)
    t0 = time.perf_counter()
    px = ref.lib.rbref_render_strided(0, 1, cores, probe_stride // 2, probe_stride)
    dt = max(time.perf_counter() - t0, 1e-3)
    assert px > 0, px
    budget = max(1.0, target_s * px / dt)            # pixel-samples that fit in target_s
    rows_full = H
    spp = int(min(wl["spp"], max(1, budget // (64 * W))))  # at least 64 rows
    rows = int(min(rows_full, max(1, budget // (spp * W))))
    stride = max(1, H // rows)
    return stride // 2, stride, spp


def _render_sample(ref, cores, first, stride, spp):
    px = ref.lib.rbref_render_strided(0, spp, cores, first, stride)
    assert px > 0, px
    return px * spp


def _sample_text(wl, first, stride, spp, steps=None):
    rows = len(range(first, wl["height"], stride))
    s = (f"{wl['width']}x{rows} rows (every {stride}th row from row {first}, spread over the whole frame) "
         f"at {spp} spp")
    return s + (f" per step, {steps} steps" if steps else "")


def cpu_baseline(scene, cie, basis, luts, wl, target_s):
    ref, keep = _ref_setup(scene, cie, basis, luts)
    cores = os.cpu_count() or 1
    first, stride, spp = _strided_sample(ref, wl, cores, target_s)
    t0 = time.perf_counter()
    paths = _render_sample(ref, cores, first, stride, spp)
    dt = time.perf_counter() - t0
    del keep
    return paths / dt, cores, _sample_text(wl, first, stride, spp) + f": {paths} paths in {dt:.2f} s"


# ----------------------------------------------------------- reference arm
def run_reference(args, rank: int, world: int, wl: dict):
    if rank != 0:
        return
    scene, cie, basis, luts, tables = make_scene(wl)
    ref, keep = _ref_setup(scene, cie, basis, luts)
    cores = os.cpu_count() or 1
    first, stride, spp = _strided_sample(ref, wl, cores, args.ref_step_s)
    for _ in range(args.warmup):
        _render_sample(ref, cores, first, stride, spp)
    t0 = time.perf_counter()
    paths = 0
    for _ in range(args.steps):
        paths += _render_sample(ref, cores, first, stride, spp)
    dt = time.perf_counter() - t0
    v = paths / dt
    sample = _sample_text(wl, first, stride, spp, args.steps)
    line = {
        "metric": METRIC, "value": v, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "impl": "reference",
        "config": workload_config(scene, wl, world, tables),
        "sample_per_step": sample,
        "cpu_baseline": {"value": v, "unit": "paths/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del keep
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args, rank: int, world: int, wl: dict):
    import torch
    from ratbite_b200 import abi, lighttree, multigpu
    from ratbite_b200.rendering_interface import RenderingInterface

    W, H, SPP = wl["width"], wl["height"], wl["spp"]
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    t_setup = time.perf_counter()
    scene, cie, basis, luts, tables = make_scene(wl)
    lt = lighttree.build_for_scene(scene)
    accel = abi.RB_ACCEL_INSTANCED if args.acceleration == "instanced" else abi.RB_ACCEL_FLAT
    ri = RenderingInterface(device=local, max_paths_in_flight=args.max_paths, acceleration=accel)
    ri.load_scene(scene, luts, cie, basis, light_tree=lt)
    cache = None
    if wl.get("cached"):
        from ratbite_b200.nrc import RadianceCache
        cache = RadianceCache(device=local, seed=2)
        ri.attach_radiance_cache(cache)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    has_env = getattr(scene, "envmap", None) is not None
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    launch = scene.launch_record()
    accum_dev = torch.zeros((H, W, 4), dtype=torch.float64, device="cuda") if world > 1 else None
    offset, _ = multigpu.weak_sample_range(SPP, rank)   # disjoint Sobol sample range per rank

    def step():
        if has_env:
            ri.rebuild_environment_cdf(stream=sp)
        if world > 1:
            multigpu.render_frame(ri, accum_dev, offset, SPP, stream=stream)
        else:
            ri.render(offset, SPP, stream=sp)

    # traversal work counts (untimed): nodes / triangles per extension and shadow ray
    ri.set_stats(abi.RB_STATS_COUNT)
    step()
    counts = ri.get_stats()
    ri.set_stats(0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-timed region (per-stage CUDA events on the render stream)
    ri.set_stats(abi.RB_STATS_TIME)
    ri.get_stats()
    if cache:
        ri.cache_stats()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    stages = ri.get_stats()
    cst = ri.cache_stats() if cache else None
    ri.set_stats(0)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    paths_per_step = W * H * SPP * world
    value = paths_per_step * args.steps / (ms / 1e3)

    # ---- end to end through the public API (host copies inside the region)
    e2e_steps = max(1, args.steps // 2)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ri.prepare_data_for_rendering(launch)            # H2D: launch parameters
        if has_env:
            ri.rebuild_environment_cdf()
        multigpu.render_range(ri, offset, SPP)
        host = ri.read_accumulation()                    # D2H: FP64 accumulation
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = paths_per_step * e2e_steps / e2e_s
    st = ri.status()

    if rank == 0:
        hbm, peak_kind = peaks()
        shares = {"extend": stages.ms_extend, "surface": stages.ms_surface, "nee": stages.ms_nee,
                  "bsdf": stages.ms_bsdf, "shadow": stages.ms_shadow,
                  "generate": stages.ms_generate, "resolve": stages.ms_resolve}
        if cst:
            shares.update({"cache_infer": cst.ms_infer, "cache_train": cst.ms_train})
        total_ms = sum(shares.values())
        dom = max(("extend", "surface", "nee", "bsdf", "shadow"), key=lambda k: shares[k])
        # counts were gathered over one step
        ext_rays, sh_rays, recs = counts.extend_rays, counts.shadow_rays, counts.surface_records
        step_bytes = {
            "extend": ext_rays * EXTEND_BYTES_PER_RAY + counts.extend_nodes * NODE_BYTES
            + counts.extend_tris * TRI_BYTES,
            "shadow": sh_rays * SHADOW_BYTES_PER_RAY + counts.shadow_nodes * NODE_BYTES
            + counts.shadow_tris * TRI_BYTES,
            "surface": ext_rays * SURFACE_BYTES_PER_PATH + recs * SURFACE_BYTES_PER_RECORD,
            "nee": recs * NEE_BYTES_PER_RECORD,
            "bsdf": recs * BSDF_BYTES_PER_RECORD,
        }
        kernel_launches = {"extend": stages.launches_extend, "shadow": stages.launches_shadow,
                           "surface": stages.launches_shade, "nee": stages.launches_nee,
                           "bsdf": stages.launches_bsdf}
        kernel_names = {"extend": "kExtend", "shadow": "kShadow", "surface": "kSurface", "nee": "kNee",
                        "bsdf": "kBsdf"}
        bytes_step = step_bytes[dom]
        launches = kernel_launches[dom]
        achieved = bytes_step * args.steps / (shares[dom] / 1e3) / 1e9
        # every kernel of ours in the timed region: the wavefront kernels and
        # one env-map CDF build per step
        launches_total = (stages.launches_generate + stages.launches_extend + stages.launches_shade
                          + stages.launches_nee + stages.launches_bsdf + stages.launches_shadow
                          + stages.launches_resolve + (args.steps if has_env else 0)
                          + (cst.launches if cst else 0))
        # DRAM traffic of the dominant kernel per launch: ncu's dram bytes per
        # work unit (measured on a reduced case of this workload, see
        # profiles/traffic.json) times the units one launch processes here
        units_step = {"extend": ext_rays, "shadow": sh_rays, "surface": ext_rays, "nee": recs, "bsdf": recs}
        traffic = None
        limiter = None
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists():
            t = json.loads(tp.read_text()).get(WORKLOADS[args.workload]["name"], {}).get(kernel_names[dom])
            if t:
                traffic = t["dram_bytes_per_unit"] * units_step[dom] / max(1.0, launches / args.steps)
                # what bounds the kernel, from one ncu capture of it: the HBM
                # fraction above is an upper bound on how memory-bound it is
                limiter = t.get("limiter")
        if args.cpu_seconds > 0:
            cpu_v, cores, sample = cpu_baseline(scene, cie, basis, luts, wl, args.cpu_seconds)
        else:
            cpu_v, cores, sample = None, 0, "skipped"
        rows = None
        if world == 1 and has_env and args.rows:
            rows = reference_kernel_rows(scene.envmap, ri.accumulation_device_ptr(), W, H)
        ttr = None
        batched = None
        if world == 1 and args.workload == "scale" and (args.ttr or args.batched):
            ri.cleanup()                     # free this workload's wave before the next ones
            if args.ttr:
                ttr = time_to_rmse(device=local)
            if args.batched:
                batched = batched_jobs(args.jobs, 1, device=local)
        line = {
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": workload_config(scene, wl, world, tables),
            "setup_s": setup_s,
            "e2e": {"value": e2e_value, "unit": "paths/s", "h2d_bytes_per_step": C.sizeof(launch),
                    "d2h_bytes_per_step": W * H * 32, "steps": e2e_steps},
            "gpu_launches": int(launches_total),
            "roofline": {"kernel": kernel_names[dom], "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "bytes_per_launch": bytes_step / max(1, launches / args.steps),
                         "limiter": limiter},
            "stages_ms_per_step": {k: v / args.steps for k, v in shares.items()},
            "stage_share": {k: (v / total_ms if total_ms else None) for k, v in shares.items()},
            "kernel_gbs": {k: (step_bytes[k] * args.steps / (shares[k] / 1e3) / 1e9 if shares[k] else None)
                           for k in step_bytes},
            "rays_per_step": {"extend": ext_rays, "shadow": sh_rays, "surface_records": recs,
                              "nodes_per_extend_ray": counts.extend_nodes / max(1, ext_rays),
                              "tris_per_extend_ray": counts.extend_tris / max(1, ext_rays),
                              "nodes_per_shadow_ray": counts.shadow_nodes / max(1, sh_rays),
                              "tris_per_shadow_ray": counts.shadow_tris / max(1, sh_rays)},
            "device_status_flags": st.flags,
            "radiance_cache": ({"queries_per_step": cst.queries / args.steps, "records_per_step": cst.records / args.steps,
                                "train_steps_per_step": cst.steps / args.steps, "last_loss": cst.last_loss}
                               if cst else None),
            "clocks": clocks.summary(),
            "cpu_baseline": {"value": cpu_v, "unit": "paths/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "time_to_rmse": ttr,
            "batched_jobs": batched,
            "reference_kernels": rows,
        }
        print(json.dumps(line), flush=True)
    ri.cleanup()
    if cache:
        cache.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def reference_kernel_rows(envmap: np.ndarray, accum_ptr: int, width: int, height: int, iters: int = 20):
    """The two rows whose reference implementation is itself a CUDA kernel,
    timed head to head on this GPU: the env-map CDF build (ours:
    rb_envmap_cdf, one fused kernel; the reference: buildCDFLatLongRGB* +
    invertCDFToIndices of src/kernels/cdf.cu compiled for sm_100a and
    launched as loadEnvironmentMap does, src/core/rendering_interface.cpp:
    1374-1419) and the resolve (ours: rb_k_resolve; the reference:
    renderResolve of src/kernels/image.cu with 16x16 blocks,
    src/core/rendering_interface.cpp:1512-1532). Each launch is timed alone
    with CUDA events after overwriting a 512 MiB buffer (L2 is 126 MB), so the
    inputs come from HBM. Algorithmic bytes: CDF 16 B read + 2 B written per
    texel plus 2 B per row (9.0 MiB at 1024x512); resolve 32 B read + 4 B
    written per pixel."""
    import torch
    from ratbite_b200 import abi, color
    from ratbite_b200._native import check, load
    ref_dir = ROOT / "oracle" / "_ref"
    lib = load()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())

    def timed(fn):
        total = 0.0
        for i in range(iters + 3):
            flush.fill_(i & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            if i >= 3:
                total += a.elapsed_time(b)
        return total / iters

    out = {}
    h, w = envmap.shape[:2]
    img = torch.from_numpy(np.ascontiguousarray(envmap, np.float32)).cuda()
    scratch = torch.zeros(int(lib.rb_envmap_cdf_scratch_bytes(w, h)), dtype=torch.uint8, device="cuda")
    cond = torch.zeros(w * h, dtype=torch.int16, device="cuda")
    marg = torch.zeros(h, dtype=torch.int16, device="cuda")
    integ = torch.zeros(1, dtype=torch.float32, device="cuda")
    cdf_bytes = w * h * 18 + h * 2
    for mode, name in ((abi.RB_CDF_REFERENCE, "ours_mode0_f32_ms"), (abi.RB_CDF_FP64, "ours_mode1_f64_ms")):
        out[name] = timed(lambda: check(lib.rb_envmap_cdf(w, h, p(img), mode, p(scratch), p(cond), p(marg),
                                                          p(integ), sp), None, "rb_envmap_cdf"))
    ref_ms = None
    if (ref_dir / "libratbite_ref_cdf.so").exists():
        rl = C.CDLL(str(ref_dir / "libratbite_ref_cdf.so"))
        rl.rbrefgpu_envmap_cdf_time.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int, C.c_int, C.c_void_p, C.c_size_t]
        rl.rbrefgpu_envmap_cdf_time.restype = C.c_float
        torch.cuda.synchronize()
        ref_ms = float(rl.rbrefgpu_envmap_cdf_time(str(ref_dir / "cdf.cubin").encode(), w, h, p(img), p(cond),
                                                   p(marg), 3, iters, p(flush), flush.numel()))
    out["reference_ms"] = ref_ms
    out["bytes"] = cdf_bytes
    out["ours_mode1_gbs"] = cdf_bytes / (out["ours_mode1_f64_ms"] / 1e3) / 1e9
    out["ours_mode0_gbs"] = cdf_bytes / (out["ours_mode0_f32_ms"] / 1e3) / 1e9
    out["reference_gbs"] = cdf_bytes / (ref_ms / 1e3) / 1e9 if ref_ms and ref_ms > 0 else None
    rows = {"envmap_cdf": dict(out, size=[w, h])}

    cs = np.ascontiguousarray(color.colorspace_matrix("sRGB"), np.float32).ravel()
    scale = float(2.0 ** (0.0 - 7.0))
    rgba = torch.zeros((height, width, 4), dtype=torch.uint8, device="cuda")
    res = {"ours_ms": timed(lambda: check(lib.rb_k_resolve(width, height, cs.ctypes.data, scale,
                                                           C.c_void_p(accum_ptr), p(rgba), sp), None,
                                          "rb_k_resolve"))}
    ref_ms = None
    if (ref_dir / "libratbite_ref_image.so").exists():
        rl = C.CDLL(str(ref_dir / "libratbite_ref_image.so"))
        rl.rbrefgpu_resolve_time.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_float, C.c_void_p,
                                             C.c_int, C.c_int, C.c_void_p, C.c_size_t]
        rl.rbrefgpu_resolve_time.restype = C.c_float
        torch.cuda.synchronize()
        ref_ms = float(rl.rbrefgpu_resolve_time(str(ref_dir / "image.cubin").encode(), width, height,
                                                cs.ctypes.data, scale, C.c_void_p(accum_ptr), 3, iters, p(flush),
                                                flush.numel()))
    rbytes = width * height * 36
    res.update(reference_ms=ref_ms, bytes=rbytes, size=[width, height],
               ours_gbs=rbytes / (res["ours_ms"] / 1e3) / 1e9,
               reference_gbs=rbytes / (ref_ms / 1e3) / 1e9 if ref_ms and ref_ms > 0 else None)
    rows["resolve"] = res
    del flush
    return rows


def batched_jobs(n_jobs: int = 64, steps: int = 1, device: int = 0):
    """Batched jobs: n_jobs render jobs drawn from a seed (ratbite_b200.batch),
    the plain ones in one shared wavefront, schedule chosen by the autotuner;
    aggregate paths/s and p50 / p99 job completion latency (device events)."""
    from ratbite_b200 import batch

    t0 = time.perf_counter()
    jobs = batch.draw_jobs(seed=5, n=n_jobs)
    cie, basis, luts, tables = bench_tables()
    br = batch.BatchRenderer(jobs, device=device, tables=(cie, basis, luts))
    setup_s = time.perf_counter() - t0
    t1 = time.perf_counter()
    best, trials = br.autotune()
    tune_s = time.perf_counter() - t1
    runs = []
    with ClockSampler(device) as clocks:
        for _ in range(max(1, steps)):
            runs.append(br.run(best))
    r = min(runs, key=lambda x: x.seconds)
    sched = lambda c: {"paths_in_flight": c.max_paths, "grid_percent": c.grid_percent, "cached_streams": c.streams,
                       "cached_samples_per_call": c.chunk}
    return {
        "workload": f"batched_{len(jobs)}_jobs", "jobs": len(jobs), "value": r.paths_per_s, "unit": "paths/s",
        "seconds": r.seconds, "runs": len(runs),
        "latency_s": {"p50": r.percentile(50), "p99": r.percentile(99), "max": max(r.latencies)},
        "sides": sorted({j.side for j in jobs}), "spp_range": [min(j.spp for j in jobs), max(j.spp for j in jobs)],
        "triangles_range": [min(j.triangles for j in jobs), max(j.triangles for j in jobs)],
        "forms": {f: sum(j.form == f for j in jobs) for f in ("plain", "cached")},
        "plain_jobs": "one shared wavefront (rb_render_jobs)", "total_paths": r.total_paths,
        "schedule": sched(best),
        "autotune": [dict(sched(c), paths_per_s=v) for c, v in trials],
        "setup_s": setup_s, "autotune_s": tune_s, "host_enqueue_s": r.host_seconds, "gpu_launches": r.gpu_launches,
        "tables": tables, "clocks": clocks.summary(),
    }


def run_batched(args):
    """The batched-jobs workload as its own bench line."""
    b = batched_jobs(args.jobs, args.steps)
    line = {
        "metric": METRIC, "value": b["value"], "unit": "paths/s", "n_gpus": 1, "steps": b["runs"],
        "warmup": 1, "ms_per_step": b["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
        "config": {k: b[k] for k in ("workload", "jobs", "sides", "spp_range", "triangles_range", "forms",
                                     "total_paths", "schedule", "autotune", "plain_jobs", "tables")},
        "latency_s": b["latency_s"], "host_enqueue_s": b["host_enqueue_s"], "gpu_launches": b["gpu_launches"],
        "clocks": b["clocks"],
    }
    print(json.dumps(line), flush=True)


def time_to_rmse(device: int = 0, width: int = 1920, height: int = 1080, depth: int = 12, ref_spp: int = 4096,
                 plain_spp: int = 1024, chunk: int = 32, failed_mode: int = 0, cache_kw: dict | None = None,
                 time_factor: float = 2.0, repeats: int = 3):
    """The cached form against the plain tracer on the Cornell box at
    width x height, depth `depth`: device seconds until each reaches the
    plain tracer's plain_spp RMSE against the FP64 oracle.

    Oracle: two independent plain renders of ref_spp samples each (FP64
    accumulation, sample indices disjoint from each other and from every
    timed run), averaged; the oracle's own noise, estimated per pixel from
    the two halves (E[(A - B)^2] / 4 is the variance of their mean), is
    subtracted from every mean squared error, so the RMSEs compared are those
    against the converged image. RMSE is taken on the linear XYZ mean image,
    relative to the oracle's mean, between chunks and outside the timed
    spans. The comparison runs `repeats` times (different sample ranges, a
    fresh untrained cache with a different seed each time); the line reports
    every ratio and their median. Both forms get one untimed warm-up chunk
    per run (first-launch costs and buffer allocation; the cache is then
    reset to its initial parameters); the cached form stops at the target or
    at time_factor x the plain tracer's time."""
    import torch
    from ratbite_b200 import lighttree, scenes
    from ratbite_b200.nrc import RadianceCache
    from ratbite_b200.rendering_interface import RenderingInterface

    cie, basis, luts, _ = bench_tables()
    scene = scenes.cornell_box(seed=1, cie_xyz=cie, width=width, height=height, spp=plain_spp, max_depth=depth)
    lt = lighttree.build_for_scene(scene)
    ri = RenderingInterface(device=device, failed_sample_mode=failed_mode)
    ri.load_scene(scene, luts, cie, basis, light_tree=lt)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    n = width * height

    def mean_image():
        ri.synchronize()
        acc = torch.from_numpy(ri.read_accumulation().reshape(n, 4)).cuda()
        return acc[:, :3] / acc[:, 3:4].clamp_min(1.0)

    ri.clear_accumulation(stream=sp)
    ri.render(1 << 24, ref_spp, stream=sp)
    half_a = mean_image()
    ri.clear_accumulation(stream=sp)
    ri.render((1 << 24) + ref_spp, ref_spp, stream=sp)
    half_b = mean_image()
    ref = 0.5 * (half_a + half_b)
    ref_mean = float(ref.mean())
    ref_noise = float(((half_a - half_b) ** 2).mean() / 4.0)       # per-pixel variance of the mean, averaged
    # pixels that see the emitter directly: the brightest 0.5 % of the oracle
    lum = ref[:, 1]
    lit = lum >= torch.quantile(lum[::97].float(), 0.995)

    def rel_rmse(img):
        mse = float(((img - ref) ** 2).mean()) - ref_noise
        return math.sqrt(max(mse, 0.0)) / ref_mean

    def biases(img):
        return (float(img.mean() / ref.mean() - 1.0), float(img[lit].mean() / ref[lit].mean() - 1.0))

    def timed(offset, count):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ri.render(offset, count, stream=sp)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / 1e3

    runs = []
    kw = dict(cache_kw or {})
    for rep in range(repeats):
        base = rep << 20                        # disjoint sample ranges per repetition
        ri.attach_radiance_cache(None)
        ri.clear_accumulation(stream=sp)
        ri.render(base + (1 << 19), chunk, stream=sp)                    # warm-up
        ri.clear_accumulation(stream=sp)
        plain_curve, t = [], 0.0
        for k in range(plain_spp // chunk):
            t += timed(base + k * chunk, chunk)
            plain_curve.append(((k + 1) * chunk, t, rel_rmse(mean_image())))
        target, t_plain = plain_curve[-1][2], plain_curve[-1][1]
        plain_bias = biases(mean_image())

        # warm-up with the cache that is then timed: it sizes the context's
        # cache buffers and the network's training scratch; the network then
        # goes back to its initial parameters (optimiser state reset) and is
        # attached again (corrections reset), so the timed run starts from an
        # untrained cache with nothing left to allocate
        cache = RadianceCache(device=device, seed=2 + rep)
        init = cache.parameters()
        ri.attach_radiance_cache(cache, **kw)
        ri.clear_accumulation(stream=sp)
        ri.render(base + (1 << 19) + chunk, chunk, stream=sp)
        ri.synchronize()
        cache.set_parameters(*init)
        ri.attach_radiance_cache(cache, **kw)
        ri.cache_stats()
        ri.clear_accumulation(stream=sp)
        cached_curve, t, done, reached = [], 0.0, 0, None
        while t < time_factor * t_plain:
            t += timed(base + (1 << 18) + done, chunk)
            done += chunk
            r = rel_rmse(mean_image())
            cached_curve.append((done, t, r))
            if r <= target:
                reached = t
                break
        st = ri.cache_stats()
        cached_bias = biases(mean_image())
        ri.attach_radiance_cache(None)
        cache.close()
        best = min(cached_curve, key=lambda c: c[2])
        runs.append({
            "plain": {"spp": plain_spp, "s": t_plain, "rel_rmse": target, "paths_per_s": n * plain_spp / t_plain,
                      "bias_image": plain_bias[0], "bias_lit_pixels": plain_bias[1]},
            "cached": {"s_to_target": reached, "spp_to_target": done if reached else None,
                       "best_rel_rmse": best[2], "best_at_spp": best[0], "spp_rendered": done, "s_rendered": t,
                       "paths_per_s": n * done / t, "queries_per_sample": st.queries / max(1, done),
                       "records_per_sample": st.records / max(1, done), "train_steps": st.steps,
                       "last_loss": st.last_loss, "bias_image": cached_bias[0], "bias_lit_pixels": cached_bias[1]},
            "time_ratio": (reached / t_plain) if reached else None,
            "plain_curve": [(a, round(b, 4), round(c, 5)) for a, b, c in plain_curve[::max(1, len(plain_curve) // 6)]],
            "cached_curve": [(a, round(b, 4), round(c, 5)) for a, b, c in cached_curve[::max(1, len(cached_curve) // 6)]],
        })
    ri.cleanup()
    ratios = [r["time_ratio"] for r in runs]
    done_ratios = sorted(x if x is not None else float("inf") for x in ratios)
    med = done_ratios[len(done_ratios) // 2]
    return {
        "workload": f"cornell_box_{width}x{height}_depth{depth}",
        "rmse": (f"relative RMSE of the XYZ mean image vs the mean of two {ref_spp}-spp FP64-accumulated plain "
                 f"renders, the oracle's own noise ({math.sqrt(ref_noise) / ref_mean:.4f} relative) subtracted"),
        "failed_sample_mode": "keep" if failed_mode else "drop (reference)",
        "params": kw or "library defaults",
        "repeats": repeats,
        "time_ratios": ratios,
        "time_ratio": med if math.isfinite(med) else None,
        "time_ratio_spread": [done_ratios[0], done_ratios[-1]] if all(map(math.isfinite, done_ratios)) else None,
        "runs": runs,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched"], default="scale")
    ap.add_argument("--jobs", type=int, default=64, help="batched workload: number of jobs")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample length (0 = skip)")
    ap.add_argument("--ref-step-s", type=float, default=4.0, help="reference arm: seconds per step")
    ap.add_argument("--spp", type=int, default=0, help="samples per pixel per step (0 = the workload's)")
    ap.add_argument("--no-ttr", dest="ttr", action="store_false",
                    help="skip the time-to-RMSE measurement of the cached form (1920x1080 Cornell box, ~30 s)")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the batched-jobs measurement (64 jobs in one shared wavefront, ~1 min)")
    ap.add_argument("--no-rows", dest="rows", action="store_false",
                    help="skip the head-to-head timing of the env-map CDF and resolve kernels against the "
                         "reference's own CUDA kernels")
    ap.add_argument("--acceleration", choices=["flat", "instanced"], default="flat",
                    help="ray-traversal structure (rb_config.acceleration): one flattened BVH (the default) or "
                         "the two-level one (a BVH per unique mesh under a top level over the instances)")
    ap.add_argument("--max-paths", type=int, default=0,
                    help="paths in flight per wave (0 = the library default, 16M); small values make profiling "
                         "captures small")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    args.warmup = max(args.warmup, 3)
    wl = dict(WORKLOADS.get(args.workload, WORKLOADS["scale"]))
    wl["acceleration"] = args.acceleration
    if args.spp:
        wl["spp"] = args.spp
        wl["name"] = wl["name"].replace(f"{WORKLOADS[args.workload]['spp']}spp", f"{args.spp}spp")
    if args.workload == "batched":
        if rank == 0 and args.impl == "ours":
            run_batched(args)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference renders one scene at a time; "
                              "batched jobs have no reference counterpart"}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world, wl)
    else:
        run_ours(args, rank, world, wl)


if __name__ == "__main__":
    main()
