"""Benchmark of the per-sample rendering path on B200.

Workload (the small plain-method configuration): seeded Cornell box, 2,574
triangles, 256x256 pixels, 64 samples per pixel, max depth 8, 4 hero
wavelengths. One step renders the whole 64-spp frame (4,194,304 paths);
metric = paths per second (higher is better).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       renders through the C ABI (libratbite_b200.so). `value` is device
           time (CUDA events on the render stream, max over ranks); `e2e` is
           the same metric through the public API with the per-step launch
           parameters uploaded and the FP64 accumulation buffer read back to
           host memory inside the timed region.
reference  the reference's own per-sample code compiled host-side
           (oracle/_ref) rendering the same scene on all host cores; each step
           renders a bounded number of samples of the same frame.

With N GPUs (torchrun) each rank renders its own 64-spp sample range of the
frame (weak scaling; Sobol indices are disjoint) and the FP64 images are
summed with one NCCL all-reduce per step, the combine step of progressive
rendering across devices.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, SPP, DEPTH = 256, 256, 64, 8
METRIC = "paths/s"
WORKLOAD = "cornell_box_256x256_64spp_depth8"


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

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
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
        for l in getattr(self, "lines", []):
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


def make_scene():
    from ratbite_b200 import assets, scenes
    cie = assets.cie_xyz()
    basis = assets.basis_rgb()
    luts = assets.luts()
    scene = scenes.cornell_box(seed=1, cie_xyz=cie, width=W, height=H, spp=SPP, max_depth=DEPTH)
    return scene, cie, basis, luts


def build_light_tree(scene):
    from ratbite_b200 import lighttree
    return lighttree.build_for_scene(scene)


# ------------------------------------------------------------- CPU baseline
def cpu_render(scene, cie, basis, luts, target_s: float, threads: int = 0):
    """Times the reference's code (oracle/_ref) on the host cores on a
    bounded sample of the frame; returns (paths/s, cores, sample text)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import RefLib, load_scene_into_ref
    ref = RefLib()
    keep = load_scene_into_ref(ref, scene, luts, cie, basis)
    cores = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    ref.lib.rbref_render(0, 1, cores)
    dt1 = max(time.perf_counter() - t0, 1e-3)
    spp = int(max(1, min(SPP, round(target_s / dt1))))
    t0 = time.perf_counter()
    ref.lib.rbref_render(0, spp, cores)
    dt = time.perf_counter() - t0
    paths = W * H * spp
    del keep
    return paths / dt, cores, f"{W}x{H} at {spp} spp ({paths} paths, {dt:.2f} s)"


# ----------------------------------------------------------- reference arm
def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    scene, cie, basis, luts = make_scene()
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import RefLib, load_scene_into_ref
    ref = RefLib()
    keep = load_scene_into_ref(ref, scene, luts, cie, basis)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref.lib.rbref_render(0, 1, cores)
    dt1 = max(time.perf_counter() - t0, 1e-3)
    spp = int(max(1, min(SPP, round(args.ref_step_s / dt1))))
    for i in range(args.warmup):
        ref.lib.rbref_render(0, spp, cores)
    t0 = time.perf_counter()
    for i in range(args.steps):
        ref.lib.rbref_render(0, spp, cores)
    dt = time.perf_counter() - t0
    paths = W * H * spp * args.steps
    v = paths / dt
    line = {
        "metric": METRIC, "value": v, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp_per_step": spp,
                   "max_depth": DEPTH, "triangles": scene.triangle_count()},
        "cpu_baseline": {"value": v, "unit": "paths/s", "cores": cores, "kind": "reference",
                         "sample": f"{W}x{H} at {spp} spp per step, {args.steps} steps"},
        "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del keep
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args, rank: int, world: int):
    import torch
    from ratbite_b200 import abi
    from ratbite_b200.rendering_interface import RenderingInterface

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    scene, cie, basis, luts = make_scene()
    lt = build_light_tree(scene)
    ri = RenderingInterface(device=local)
    ri.load_scene(scene, luts, cie, basis, light_tree=lt)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    launch = scene.launch_record()
    accum_dev = torch.zeros((H, W, 4), dtype=torch.float64, device="cuda")
    offset = rank * SPP                     # disjoint Sobol sample range per rank

    def step():
        ri.render(offset, SPP, stream=sp)
        if world > 1:
            ri.copy_accumulation_async(accum_dev.data_ptr(), stream=sp)
            with torch.cuda.stream(stream):
                dist.all_reduce(accum_dev)

    # traversal work counts (untimed): nodes / triangles per extension and shadow ray
    ri.set_stats(abi.RB_STATS_COUNT)
    step()
    counts = ri.get_stats()
    ri.set_stats(0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-timed region (per-stage events on the render stream)
    ri.set_stats(abi.RB_STATS_TIME)
    ri.get_stats()
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
    ri.set_stats(0)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    paths_per_step = W * H * SPP * world
    value = paths_per_step * args.steps / (ms / 1e3)

    # ---- end to end through the public API (host copies inside the region)
    host = np.zeros((H, W, 4), np.float64)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ri.prepare_data_for_rendering(launch)            # H2D: launch parameters
        ri.render(offset, SPP)
        host = ri.read_accumulation()                    # D2H: FP64 accumulation
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = paths_per_step * args.steps / e2e_s
    st = ri.status()

    if rank == 0:
        # Roofline of the dominant stage (HBM-bound model; bytes per unit in DESIGN.md).
        hbm, peak_kind = peaks()
        shares = {"extend": stages.ms_extend, "shade": stages.ms_shade, "shadow": stages.ms_shadow,
                  "generate": stages.ms_generate, "resolve": stages.ms_resolve}
        total_ms = sum(shares.values())
        dom = max(("extend", "shade", "shadow"), key=lambda k: shares[k])
        per_step = lambda x: x / max(1, counts.waves)          # counts were gathered over one step
        ext_rays = per_step(counts.extend_rays)
        sh_rays = per_step(counts.shadow_rays)
        if dom == "extend":
            bytes_step = ext_rays * (32 + 16) + per_step(counts.extend_nodes) * 96 + per_step(counts.extend_tris) * 48
            launches = stages.launches_extend
        elif dom == "shadow":
            bytes_step = sh_rays * (32 + 4) + per_step(counts.shadow_nodes) * 96 + per_step(counts.shadow_tris) * 48
            launches = stages.launches_shadow
        else:
            bytes_step = ext_rays * SHADE_BYTES_PER_PATH
            launches = stages.launches_shade
        stage_ms = shares[dom]
        achieved = bytes_step * args.steps / (stage_ms / 1e3) / 1e9
        launches_per_step = (stages.launches_generate + stages.launches_extend + stages.launches_shade
                             + stages.launches_shadow + stages.launches_resolve) / args.steps
        traffic = None
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists():
            traffic = json.loads(tp.read_text()).get(dom)
        cpu_v, cores, sample = cpu_render(scene, cie, basis, luts, args.cpu_seconds) if args.cpu_seconds > 0 else (None, 0, "skipped")
        line = {
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "max_depth": DEPTH,
                       "triangles": scene.triangle_count(), "paths_per_step": paths_per_step,
                       "parallelism": f"sample-range x{world}",
                       "l2": "inputs larger than L2 (wavefront path state ~800 MB per wave)"},
            "e2e": {"value": e2e_value, "unit": "paths/s", "h2d_bytes_per_step": C.sizeof(launch),
                    "d2h_bytes_per_step": W * H * 32},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "bytes_per_launch": bytes_step / max(1, launches / args.steps)},
            "stages_ms_per_step": {k: v / args.steps for k, v in shares.items()},
            "stage_share": {k: (v / total_ms if total_ms else None) for k, v in shares.items()},
            "rays_per_step": {"extend": ext_rays, "shadow": sh_rays,
                              "nodes_per_extend_ray": counts.extend_nodes / max(1, counts.extend_rays),
                              "tris_per_extend_ray": counts.extend_tris / max(1, counts.extend_rays)},
            "device_status_flags": st.flags,
            "clocks": clocks.summary(),
            "cpu_baseline": {"value": cpu_v, "unit": "paths/s", "cores": cores, "kind": "reference",
                             "sample": sample},
        }
        print(json.dumps(line), flush=True)
    ri.cleanup()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# Algorithmic bytes of one shading step (kShade) per path: path state read and
# written (ray o/d, wavelengths, pdfs, normal, L, T: 7 x 16 B, twice), flags,
# the hit record, the hit triangle (3 x 16 B + 8 B), the material record
# (128 B), the vertex indices and 3 attribute reads (6 + 24 B), LUT taps (two
# 3D tables x 8 taps + one 2D x 4 taps, 4 B each), spectral basis and sensor
# lookups (12 x 4 B), the emitter record (68 B) and the shadow request written
# (48 B). Light-tree node reads grow with tree depth and are not counted.
SHADE_BYTES_PER_PATH = 2 * 7 * 16 + 2 * 8 + 16 + 56 + 128 + 30 + 20 * 4 + 12 * 4 + 68 + 48


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample length (0 = skip)")
    ap.add_argument("--ref-step-s", type=float, default=4.0, help="reference arm: seconds per step")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
