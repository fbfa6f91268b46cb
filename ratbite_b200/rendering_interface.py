"""Host-side mirror of ratbite's RenderingInterface
(src/core/rendering_interface.h:19-226) over the B200 C ABI.

Method names follow the reference where they have a counterpart:
loadLookUpTables / fillSpectralCurvesData / fillModelMaterials /
loadModel (geometry) / loadLights / loadEnvironmentMap / prepareDataForRendering
/ render. The object owns one rb_ctx; all device memory belongs to it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._native import check, load, stream_arg


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class RenderingInterface:
    def __init__(self, device: int = 0, max_paths_in_flight: int = 0, envmap_cdf_mode: int = abi.RB_CDF_FP64,
                 failed_sample_mode: int = abi.RB_FAILED_DROP, inject: dict | None = None,
                 acceleration: int = abi.RB_ACCEL_FLAT):
        """inject: fault injection for tests, keys of rb_config without the
        `inject_` prefix (queue_limit, alloc_failure, stack_limit).
        acceleration: RB_ACCEL_FLAT or RB_ACCEL_INSTANCED (two-level)."""
        self.lib = load()
        cfg = abi.rb_config()
        cfg.device = device
        cfg.max_paths_in_flight = max_paths_in_flight
        cfg.envmap_cdf_mode = envmap_cdf_mode
        cfg.failed_sample_mode = failed_sample_mode
        cfg.acceleration = acceleration
        for k, v in (inject or {}).items():
            setattr(cfg, f"inject_{k}", int(v))
        h = C.c_void_p()
        check(self.lib.rb_create(C.byref(cfg), C.byref(h)), None, "rb_create")
        self.ctx = h
        self.width = self.height = 0
        self._keep = []
        self._cache = None

    # ---- lifetime ----------------------------------------------------------
    def cleanup(self):
        if self.ctx:
            self.lib.rb_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.cleanup()

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    # ---- uploads -----------------------------------------------------------
    def load_look_up_tables(self, luts: dict):
        arrs = [np.ascontiguousarray(luts[k], np.float32) for k in
                ("conductor", "dielectric_outer", "dielectric_inner", "reflective_outer",
                 "reflective_inner", "sheen")]
        sizes = [32 * 32, 32 ** 3, 32 ** 3, 32 ** 3, 32 ** 3, 32 * 32 * 4]
        for a, s in zip(arrs, sizes):
            if a.size != s:
                raise ValueError(f"LUT has {a.size} values, expected {s}")
        check(self.lib.rb_set_luts(self.ctx, *[_ptr(a) for a in arrs]), self.ctx, "rb_set_luts")

    def fill_spectral_curves_data(self, sensor_xyz: np.ndarray, basis_rgb: np.ndarray,
                                  extra: np.ndarray | None = None):
        s = np.ascontiguousarray(sensor_xyz, np.float32).reshape(3, abi.RB_SPECTRUM_BINS)
        b = np.ascontiguousarray(basis_rgb, np.float32).reshape(3, abi.RB_SPECTRUM_BINS)
        e = (np.zeros((0, abi.RB_SPECTRUM_BINS), np.float32) if extra is None
             else np.ascontiguousarray(extra, np.float32).reshape(-1, abi.RB_SPECTRUM_BINS))
        check(self.lib.rb_set_spectra(self.ctx, _ptr(s), _ptr(b), _ptr(e) if len(e) else None, len(e)),
              self.ctx, "rb_set_spectra")

    def load_textures(self, records):
        check(self.lib.rb_set_textures(self.ctx, C.cast(records, C.c_void_p), len(records)),
              self.ctx, "rb_set_textures")

    def fill_model_materials(self, records):
        check(self.lib.rb_set_materials(self.ctx, C.cast(records, C.c_void_p), len(records)),
              self.ctx, "rb_set_materials")

    def load_geometry(self, geometry: abi.rb_geometry):
        check(self.lib.rb_set_geometry(self.ctx, C.byref(geometry)), self.ctx, "rb_set_geometry")

    def load_lights(self, light_tree: abi.rb_light_tree):
        check(self.lib.rb_set_lights(self.ctx, C.byref(light_tree)), self.ctx, "rb_set_lights")

    def load_environment_map(self, rgba: np.ndarray):
        img = np.ascontiguousarray(rgba, np.float32)
        h, w = img.shape[:2]
        check(self.lib.rb_set_envmap(self.ctx, _ptr(img), w, h), self.ctx, "rb_set_envmap")

    def rebuild_environment_cdf(self, stream=None):
        s = stream_arg(stream)
        check(self.lib.rb_rebuild_envmap_cdf(self.ctx, s), self.ctx, "rb_rebuild_envmap_cdf")

    def clear_environment_map(self):
        check(self.lib.rb_clear_envmap(self.ctx), self.ctx, "rb_clear_envmap")

    def prepare_data_for_rendering(self, launch: abi.rb_launch):
        check(self.lib.rb_set_launch(self.ctx, C.byref(launch)), self.ctx, "rb_set_launch")
        self.width, self.height = launch.width, launch.height

    def load_scene(self, scene, luts: dict, sensor_xyz, basis_rgb, light_tree=None, extra=None,
                   width=None, height=None, max_depth=None):
        """Uploads a ratbite_b200.scenes.Scene (and its light tree records)."""
        self.load_look_up_tables(luts)
        self.fill_spectral_curves_data(sensor_xyz, basis_rgb, extra)
        texs = scene.texture_records()
        self._keep.append(texs)
        self.load_textures(texs)
        mats = scene.material_records()
        self._keep.append(mats)
        self.fill_model_materials(mats)
        g = scene.geometry_record()
        self._keep.append(g)
        self.load_geometry(g)
        if light_tree is not None:
            self._keep.append(light_tree)
            self.load_lights(light_tree)
        env = getattr(scene, "envmap", None)
        if env is not None:
            self.load_environment_map(env)
        launch = scene.launch_record(width, height, max_depth)
        self._keep.append(launch)
        self.prepare_data_for_rendering(launch)

    def build_lights(self, world, flux, material, primitive, uvs=None, stream=None):
        """Builds the light tree on the device (rb_build_lights) from the
        emissive triangles (host arrays, uploaded first; `uvs`, (n, 6), the
        emission texture's coordinates per triangle, e.g. Scene.emissive_uvs)
        and installs it."""
        import torch
        n = len(flux)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        bufs = [dev(np.asarray(world, np.float32).reshape(n, 9)), dev(np.asarray(flux, np.float32)),
                dev(np.asarray(material, np.uint32).view(np.int32)), dev(np.asarray(primitive, np.uint32).view(np.int32))]
        uv = None if uvs is None else dev(np.asarray(uvs, np.float32).reshape(n, 6))
        torch.cuda.synchronize()
        ptrs = [C.c_void_p(b.data_ptr()) for b in bufs] + [None if uv is None else C.c_void_p(uv.data_ptr())]
        check(self.lib.rb_build_lights(self.ctx, n, *ptrs, stream_arg(stream)), self.ctx, "rb_build_lights")

    def update_instances(self, instance_transforms, subset_transforms=None, stream=None):
        """Moves the instances of the loaded geometry (the reference's
        updateInstanceAccelerationStructure on a camera move): (n, 3, 4)
        camera-relative transforms in the order of the scene's instances and
        emissive subsets; the BVH is refit on the device."""
        inst = np.ascontiguousarray(instance_transforms, np.float32).reshape(-1)
        sub = np.ascontiguousarray(np.zeros(0, np.float32) if subset_transforms is None else subset_transforms,
                                   np.float32).reshape(-1)
        s = stream_arg(stream)
        check(self.lib.rb_update_instances(self.ctx, _ptr(inst) if inst.size else None,
                                           _ptr(sub) if sub.size else None, s), self.ctx, "rb_update_instances")

    def set_light_origin(self, origin, stream=None):
        """Camera-move refresh of the light data on the device: emissive
        triangle vertices and light-tree means become (as loaded) - origin."""
        o = np.ascontiguousarray(origin, np.float32).reshape(3)
        s = stream_arg(stream)
        check(self.lib.rb_set_light_origin(self.ctx, _ptr(o), s), self.ctx, "rb_set_light_origin")

    # ---- rendering -----------------------------------------------------------
    def render(self, sample_offset: int, sample_count: int, stream=None):
        """Asynchronous: renders samples [offset, offset+count) of every pixel."""
        s = stream_arg(stream)
        check(self.lib.rb_render(self.ctx, sample_offset, sample_count, s), self.ctx, "rb_render")

    def render_graph(self, sample_offset: int, sample_count: int, stream=None):
        """render() through a captured CUDA graph of the call's waves (same
        accumulation); the first call of a sample count captures it."""
        s = stream_arg(stream)
        check(self.lib.rb_render_graph(self.ctx, sample_offset, sample_count, s), self.ctx, "rb_render_graph")

    def progressive_restart(self, total_samples: int, mode: int = abi.RB_MODE_GRADUAL):
        """Restarts the progressive render (the next step renders sample 0 alone)."""
        check(self.lib.rb_progressive_restart(self.ctx, total_samples, mode), self.ctx, "rb_progressive_restart")

    def progressive_step(self, stream=None) -> abi.rb_progress:
        """Launches the next sub-launch of the progressive render (asynchronous)."""
        out = abi.rb_progress()
        s = stream_arg(stream)
        check(self.lib.rb_progressive_step(self.ctx, s, C.byref(out)), self.ctx, "rb_progressive_step")
        return out

    def synchronize(self):
        check(self.lib.rb_synchronize(self.ctx), self.ctx, "rb_synchronize")

    def read_accumulation(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float64)
        check(self.lib.rb_read_accum(self.ctx, _ptr(out)), self.ctx, "rb_read_accum")
        return out

    def write_accumulation(self, accum: np.ndarray):
        """Overwrites the accumulation buffer (rb_write_accum)."""
        a = np.ascontiguousarray(accum, np.float64)
        if a.shape != (self.height, self.width, 4):
            raise ValueError(f"accumulation is {a.shape}, the film is {(self.height, self.width, 4)}")
        check(self.lib.rb_write_accum(self.ctx, _ptr(a)), self.ctx, "rb_write_accum")

    def save_checkpoint(self, path, next_offset: int, cache=None):
        """Writes what resumes this render (np.savez): the FP64
        accumulation, the next sample offset and the film size, and with a
        radiance cache its parameters (grid and weights; the optimiser's
        moments restart on resume)."""
        extra = {}
        if cache is not None:
            grid, weights = cache.parameters()
            extra = dict(cache_grid=grid, cache_weights=weights)
        np.savez(path, accum=self.read_accumulation(), next_offset=np.int64(next_offset),
                 film=np.array([self.width, self.height], np.int64), **extra)

    def load_checkpoint(self, path, cache=None) -> int:
        """Restores a checkpoint of save_checkpoint into this context (scene
        and launch already loaded, same film) and returns the next sample
        offset: rendering on from it adds to the restored accumulation
        exactly as the interrupted render would have."""
        with np.load(path) as z:
            if tuple(int(v) for v in z["film"]) != (self.width, self.height):
                raise ValueError("checkpoint film size differs from the loaded launch")
            self.write_accumulation(z["accum"])
            if cache is not None and "cache_grid" in z:
                cache.set_parameters(z["cache_grid"], z["cache_weights"])
            return int(z["next_offset"])

    def copy_accumulation_async(self, dst_ptr: int, stream=None):
        """Stream-ordered copy into device or pinned host memory at dst_ptr."""
        s = stream_arg(stream)
        check(self.lib.rb_copy_accum_async(self.ctx, C.c_void_p(dst_ptr), s), self.ctx, "rb_copy_accum_async")

    def resolve(self, exposure: float = 0.0, colorspace=None, stream=None):
        """Resolves the accumulation into the headless RGBA8 image (stream-ordered):
        AgX tonemap with exposure scale 2^(exposure - 7), as the reference's
        resolveRender. `colorspace`: 9 floats, column-major XYZ -> RGB (default sRGB)."""
        from .color import colorspace_matrix
        cs = colorspace_matrix("sRGB") if colorspace is None else np.ascontiguousarray(colorspace, np.float32)
        if cs.size != 9:
            raise ValueError("colorspace must hold 9 floats")
        s = stream_arg(stream)
        check(self.lib.rb_resolve(self.ctx, _ptr(cs), float(2.0 ** (exposure - 7.0)), s), self.ctx, "rb_resolve")

    def read_image(self) -> np.ndarray:
        """The resolved image as an (H, W, 4) uint8 array (synchronizes)."""
        out = np.zeros((self.height, self.width, 4), np.uint8)
        check(self.lib.rb_read_image(self.ctx, _ptr(out)), self.ctx, "rb_read_image")
        return out

    def clear_accumulation(self, stream=None):
        """Zeroes the FP64 accumulation (stream-ordered)."""
        s = stream_arg(stream)
        check(self.lib.rb_clear_accum(self.ctx, s), self.ctx, "rb_clear_accum")

    def accumulation_device_ptr(self) -> int:
        p = C.c_void_p()
        check(self.lib.rb_accum_device_ptr(self.ctx, C.byref(p)), self.ctx, "rb_accum_device_ptr")
        return p.value

    def set_stats(self, mode: int):
        check(self.lib.rb_set_stats(self.ctx, mode), self.ctx, "rb_set_stats")

    def get_stats(self) -> abi.rb_render_stats:
        st = abi.rb_render_stats()
        check(self.lib.rb_get_stats(self.ctx, C.byref(st)), self.ctx, "rb_get_stats")
        return st

    def status(self) -> abi.rb_device_status:
        st = abi.rb_device_status()
        check(self.lib.rb_status(self.ctx, C.byref(st)), self.ctx, "rb_status")
        return st

    # ---- radiance-cache form (include/ratbite_b200_nrc.h) -------------------
    def attach_radiance_cache(self, cache, spread_threshold: float = 0.0, train_one_in: int = 0,
                              targets_per_sample: int = 0, batch: int = 0, frozen: bool = False,
                              samples_per_wave: int = 0, scene_bounds=None, min_roughness: float = 0.0):
        """Renders through `cache` (a RadianceCache, or None to detach);
        zero arguments take the library's defaults."""
        if cache is None:
            check(self.lib.rb_attach_radiance_cache(self.ctx, None, None), self.ctx, "rb_attach_radiance_cache")
            self._cache = None
            return
        p = abi.rb_cache_params()
        p.spread_threshold = spread_threshold
        p.train_one_in = train_one_in
        p.targets_per_sample = targets_per_sample
        p.batch = batch
        p.frozen = 1 if frozen else 0
        p.samples_per_wave = samples_per_wave
        p.min_roughness = min_roughness
        if scene_bounds is not None:
            lo, hi = scene_bounds
            p.scene_min[:] = [float(v) for v in lo]
            p.scene_max[:] = [float(v) for v in hi]
        check(self.lib.rb_attach_radiance_cache(self.ctx, cache.h, C.byref(p)), self.ctx,
              "rb_attach_radiance_cache")
        self._cache = cache   # the cache must outlive the attachment

    def cache_stats(self) -> abi.rb_cache_stats:
        """What the cached form gathered since the last call (queries,
        training records, optimiser steps, latest loss, launches, stage times)
        and the corrections it currently applies: drop_bias and
        drop_bias_other (added to the predicted drop probability of queries
        whose camera ray hit an emitter, and of the others) and
        radiance_scale. Synchronizes; the counters restart."""
        st = abi.rb_cache_stats()
        check(self.lib.rb_get_cache_stats(self.ctx, C.byref(st)), self.ctx, "rb_get_cache_stats")
        return st


def render_jobs(interfaces, offsets, counts, max_paths: int = 0, grid_percent: int = 0, done_events=None,
                stream=None):
    """Renders several RenderingInterface jobs in one shared wavefront
    (rb_render_jobs): job j renders samples [offsets[j], offsets[j] +
    counts[j]). done_events: optional torch.cuda.Event per job, recorded when
    the job's last wave completes."""
    lib = load()
    n = len(interfaces)
    ctxs = (C.c_void_p * n)(*[ri.ctx.value for ri in interfaces])
    offs = (C.c_uint32 * n)(*offsets)
    cnts = (C.c_uint32 * n)(*counts)
    opt = abi.rb_jobs_options()
    opt.max_paths_in_flight = max_paths
    opt.grid_percent = grid_percent
    ev = None
    if done_events is not None:
        ev = (C.c_void_p * n)(*[e.cuda_event if e is not None else None for e in done_events])
        opt.done_events = C.cast(ev, C.c_void_p)
    check(lib.rb_render_jobs(ctxs, n, offs, cnts, C.byref(opt), stream_arg(stream)), interfaces[0].ctx,
          "rb_render_jobs")
