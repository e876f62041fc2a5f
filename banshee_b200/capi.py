"""ctypes binding of libbanshee_gpu.so (include/banshee_gpu.h).

There is no fallback: if the shared library is missing or no sm_100 device is
present, constructing a Context raises.  Device buffers are torch CUDA tensors
(torch supplies device memory and streams only; all compute runs in the
library's own kernels).
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbanshee_gpu.so")

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_lib = None


class BansheeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (abi.BG_ERR.get(code, "BG_ERR"), code, msg))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbanshee_gpu.so is not built (%s); run banshee_b200/build.py" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.bg_last_error.restype = C.c_char_p
        sig = {
            "bg_version": [C.POINTER(_i32), C.POINTER(_i32)],
            "bg_ctx_create": [_i32, C.POINTER(_vp)],
            "bg_ctx_destroy": [_vp],
            "bg_ctx_sync": [_vp],
            "bg_scene_create": [_vp, C.POINTER(_vp)],
            "bg_scene_destroy": [_vp],
            "bg_scene_add_mesh": [_vp, C.POINTER(abi.MeshDesc), C.POINTER(_i32)],
            "bg_scene_add_material": [_vp, C.POINTER(abi.MaterialDesc), C.POINTER(_i32)],
            "bg_scene_add_light": [_vp, C.POINTER(abi.LightDesc), C.POINTER(_i32)],
            "bg_scene_set_background": [_vp, C.POINTER(C.c_float)],
            "bg_scene_commit": [_vp, C.POINTER(abi.BuildOpts)],
            "bg_scene_info_get": [_vp, C.POINTER(abi.SceneInfo)],
            "bg_scene_error_flags": [_vp, C.POINTER(C.c_uint32), _i32],
            "bg_scene_set_node_width": [_vp, _i32],
            "bg_image_finalize": [_vp, _i32, _i32, _vp],
            "bg_image_write": [C.c_char_p, _vp, _i32, _i32],
            "bg_intersect_closest": [_vp, _vp, _vp, _i64, _vp],
            "bg_intersect_any": [_vp, _vp, _vp, _i64, _vp],
            "bg_intersect_closest_host": [_vp, _vp, _vp, _i64],
            "bg_intersect_any_host": [_vp, _vp, _vp, _i64],
            "bg_traversal_counts": [_vp, _vp, _i64, _i32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _vp],
            "bg_traversal_counts_noalloc": [_vp, _vp, _i64, _i32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                            _vp],
            "bg_render": [_vp, C.POINTER(abi.CameraDesc), C.POINTER(abi.TracerDesc), C.POINTER(abi.SamplerDesc),
                          _i32, _i32, _vp, C.POINTER(abi.RenderStats), _vp],
            "bg_render_host": [_vp, C.POINTER(abi.CameraDesc), C.POINTER(abi.TracerDesc),
                               C.POINTER(abi.SamplerDesc), _i32, _i32, _vp, C.POINTER(abi.RenderStats)],
            "bg_batch_create": [_vp, C.POINTER(_vp)],
            "bg_batch_add_scene": [_vp, _vp, C.POINTER(_i32)],
            "bg_batch_commit": [_vp],
            "bg_batch_info": [_vp, C.POINTER(abi.SceneInfo)],
            "bg_batch_render": [_vp, C.POINTER(abi.BatchJob), _i32, C.POINTER(abi.TracerDesc),
                                C.POINTER(abi.RenderStats), _vp],
            "bg_batch_autotune": [_vp, C.POINTER(abi.BatchJob), _i32, C.POINTER(abi.TracerDesc), _i32,
                                  C.POINTER(abi.TuneResult), _vp],
            "bg_batch_destroy": [_vp],
            "bg_scene_autotune": [_vp, C.POINTER(abi.CameraDesc), C.POINTER(abi.TracerDesc), _i32, _i32, _i32, _vp,
                                  C.POINTER(abi.TuneResult), _vp],
            "bg_cache_create": [_vp, C.POINTER(abi.CacheDesc), C.POINTER(_vp)],
            "bg_cache_destroy": [_vp],
            "bg_cache_info": [_vp, C.POINTER(_i32), C.POINTER(_i64), C.POINTER(_i32), C.POINTER(C.c_float)],
            "bg_cache_query": [_vp, _vp, _vp, _i64, _vp],
            "bg_cache_train": [_vp, _vp, _vp, _i64, _i32, C.POINTER(C.c_float), _vp],
            "bg_cache_params": [_vp, _vp, _vp, _vp, _vp],
            "bg_cache_set_params": [_vp, _vp, _vp],
            "bg_alloc_limit": [_i64],
            "bg_alloc_stats_get": [C.POINTER(abi.AllocStats)],
            "bg_render_cached": [_vp, _vp, C.POINTER(abi.CameraDesc), C.POINTER(abi.TracerDesc),
                                 C.POINTER(abi.SamplerDesc), _i32, _i32, _vp, C.POINTER(abi.RenderStats), _vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = L
    return _lib


def check(rc):
    if rc != abi.BG_OK:
        raise BansheeError(rc, lib().bg_last_error().decode(errors="replace"))
    return rc


def _stream_handle(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(stream)


def alloc_limit(nbytes):
    """bg_alloc_limit: allow `nbytes` more bytes of library allocations from now
    on (None or a negative value removes the cap)."""
    check(lib().bg_alloc_limit(-1 if nbytes is None else int(nbytes)))


def alloc_stats():
    """bg_alloc_stats_get: allocations made / bytes / refused by the cap / budget left."""
    st = abi.AllocStats()
    check(lib().bg_alloc_stats_get(C.byref(st)))
    return {k: getattr(st, k) for k, _ in abi.AllocStats._fields_}


class Context:
    """bg_ctx: one per CUDA device."""

    def __init__(self, device=0):
        self.h = _vp()
        check(lib().bg_ctx_create(int(device), C.byref(self.h)))
        self.device = int(device)

    def sync(self):
        check(lib().bg_ctx_sync(self.h))

    def close(self):
        if self.h:
            lib().bg_ctx_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuScene:
    """A committed scene on the device: World::Commit + the Intersectable surface."""

    def __init__(self, ctx, scene, node_width=0, max_leaf=4, bins=32, builder=0, commit=True, intersect=0):
        """node_width: 4 (128-byte nodes), 8 (96-byte compressed nodes) or 0 (both
        built; the active one is chosen with set_node_width).  builder: 0 = host
        binned SAH, 1 = device LBVH, 2 = device PLOC, 3 = device binned SAH.
        commit=False leaves the scene assembled but uncommitted (commit()).
        intersect: 0 = the reference's Moller-Trumbore (bit-exact hits),
        1 = the watertight test."""
        self.ctx = ctx
        self.scene = scene
        self.h = _vp()
        L = lib()
        check(L.bg_scene_create(ctx.h, C.byref(self.h)))
        for m in scene.meshes:
            d = m.desc()
            check(L.bg_scene_add_mesh(self.h, C.byref(d), None))
        for md in scene.materials:
            from .scene import material_desc
            d = material_desc(md)
            check(L.bg_scene_add_material(self.h, C.byref(d), None))
        for ld in scene.lights:
            from .scene import light_desc
            d = light_desc(ld)
            check(L.bg_scene_add_light(self.h, C.byref(d), None))
        bg = (C.c_float * 3)(*scene.bgcolor)
        check(L.bg_scene_set_background(self.h, bg))
        self._opts = abi.BuildOpts(node_width, max_leaf, bins, builder, intersect)
        if commit:
            self.commit()

    def commit(self):
        """bg_scene_commit with the build options given at construction."""
        check(lib().bg_scene_commit(self.h, C.byref(self._opts)))

    def info(self):
        i = abi.SceneInfo()
        check(lib().bg_scene_info_get(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in abi.SceneInfo._fields_}

    def error_flags(self, clear=True):
        f = C.c_uint32()
        check(lib().bg_scene_error_flags(self.h, C.byref(f), int(clear)))
        return f.value

    def set_node_width(self, width):
        check(lib().bg_scene_set_node_width(self.h, int(width)))

    def autotune(self, accum_dev, width, height, probe_spp=1, tracer=abi.BG_TRACER_GI, maxdepth=8, camera=None,
                 stream=None):
        """bg_scene_autotune: picks node width, traversal block size and paths per pass
        for this scene and camera; accum_dev receives the probe samples."""
        cam = self.scene.camera_desc() if camera is None else camera
        tr = abi.TracerDesc(tracer, maxdepth, 0, 0.0)
        res = abi.TuneResult()
        check(lib().bg_scene_autotune(self.h, C.byref(cam), C.byref(tr), int(probe_spp), int(width), int(height),
                                      accum_dev, C.byref(res), _stream_handle(stream)))
        return {k: getattr(res, k) for k, _ in abi.TuneResult._fields_}

    # -- host-buffer entry points (synchronous) --------------------------------
    def intersect_closest_host(self, rays):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=abi.HIT_DTYPE)
        check(lib().bg_intersect_closest_host(self.h, rays.ctypes.data, hits.ctypes.data, rays.shape[0]))
        return hits

    def intersect_any_host(self, rays):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        occ = np.zeros(rays.shape[0], dtype=np.uint8)
        check(lib().bg_intersect_any_host(self.h, rays.ctypes.data, occ.ctypes.data, rays.shape[0]))
        return occ

    # -- device-buffer entry points (async on a stream) ------------------------
    def intersect_closest(self, rays_dev, hits_dev, n, stream=None):
        check(lib().bg_intersect_closest(self.h, rays_dev, hits_dev, int(n), _stream_handle(stream)))

    def intersect_any(self, rays_dev, occ_dev, n, stream=None):
        check(lib().bg_intersect_any(self.h, rays_dev, occ_dev, int(n), _stream_handle(stream)))

    def traversal_counts(self, rays_dev, n, any_hit=False, stream=None):
        a, b = C.c_uint64(), C.c_uint64()
        check(lib().bg_traversal_counts(self.h, rays_dev, int(n), int(any_hit), C.byref(a), C.byref(b),
                                        _stream_handle(stream)))
        return a.value, b.value

    def traversal_counts_noalloc(self, rays_dev, n, any_hit=False, stream=None):
        """bg_traversal_counts_noalloc: the same counts with the library's static scratch."""
        a, b = C.c_uint64(), C.c_uint64()
        check(lib().bg_traversal_counts_noalloc(self.h, rays_dev, int(n), int(any_hit), C.byref(a), C.byref(b),
                                                _stream_handle(stream)))
        return a.value, b.value

    def render(self, accum_dev, width, height, spp, seed=1, sample_offset=0, tracer=abi.BG_TRACER_GI,
               maxdepth=5, camera=None, stream=None, flags=0, stats=True, sampler=abi.BG_SAMPLER_RANDOM, grid=0,
               ao_radius=0.0):
        """Asynchronous on `stream` unless stats=True (statistics synchronize)."""
        cam = self.scene.camera_desc() if camera is None else camera
        tr = abi.TracerDesc(tracer, maxdepth, flags, ao_radius)
        sm = abi.SamplerDesc(sampler, spp, seed, sample_offset, grid)
        st = abi.RenderStats()
        check(lib().bg_render(self.h, C.byref(cam), C.byref(tr), C.byref(sm), int(width), int(height),
                              accum_dev, C.byref(st) if stats else None, _stream_handle(stream)))
        return {k: getattr(st, k) for k, _ in abi.RenderStats._fields_} if stats else None

    def render_host(self, width, height, spp, seed=1, sample_offset=0, tracer=abi.BG_TRACER_GI, maxdepth=5,
                    camera=None, accum=None, stats=None, flags=0, sampler=abi.BG_SAMPLER_RANDOM, grid=0,
                    ao_radius=0.0):
        cam = self.scene.camera_desc() if camera is None else camera
        if accum is None:
            accum = np.zeros((height, width, 4), dtype=np.float32)
        tr = abi.TracerDesc(tracer, maxdepth, flags, ao_radius)
        sm = abi.SamplerDesc(sampler, spp, seed, sample_offset, grid)
        st = abi.RenderStats()
        check(lib().bg_render_host(self.h, C.byref(cam), C.byref(tr), C.byref(sm), int(width), int(height),
                                   accum.ctypes.data, C.byref(st) if stats is not None else None))
        if stats is not None:
            stats.update({k: getattr(st, k) for k, _ in abi.RenderStats._fields_})
        return accum

    def close(self):
        if self.h:
            lib().bg_scene_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RadianceCache:
    """bg_cache: the online-trained neural radiance cache of a committed scene."""

    def __init__(self, gscene, log2_table_size=19, base_resolution=16, max_resolution=2048, train_paths=65536,
                 cache_depth=2, train_batch=16384, train_steps=4, learning_rate=1e-2, bbox=None, seed=1,
                 mlp_kernel=0, train_suffix=0, wait_polls=0):
        """mlp_kernel: inference on tcgen05 with TMEM accumulators (0) or on mma.sync (1).
        train_suffix: 0 = training paths run to maxdepth; k > 0 = they end into the
        cache k bounces after cache_depth (self-training).  wait_polls: budget of
        the tcgen05 kernels' bounded mbarrier waits (0 = default)."""
        d = abi.CacheDesc()
        d.levels = 16
        d.log2_table_size = log2_table_size
        d.base_resolution = base_resolution
        d.max_resolution = max_resolution
        d.train_paths = train_paths
        d.cache_depth = cache_depth
        d.train_batch = train_batch
        d.train_steps = train_steps
        d.learning_rate = learning_rate
        if bbox is not None:
            d.bbox_min[:] = list(bbox[0])
            d.bbox_max[:] = list(bbox[1])
        d.seed = seed
        d.mlp_kernel = mlp_kernel
        d.train_suffix = train_suffix
        d.wait_polls = wait_polls
        self.gs = gscene
        self.h = _vp()
        check(lib().bg_cache_create(gscene.h, C.byref(d), C.byref(self.h)))
        self.log2_table_size = log2_table_size

    def info(self):
        nm, ng = _i32(), _i64()
        res = (_i32 * 16)()
        norm = (C.c_float * 6)()
        check(lib().bg_cache_info(self.h, C.byref(nm), C.byref(ng), res, norm))
        return {"mlp_params": nm.value, "grid_params": ng.value, "resolutions": list(res),
                "bmin": np.array(norm[:3], dtype=np.float32), "bscale": np.array(norm[3:], dtype=np.float32)}

    def query(self, feat_dev, out_dev, n, stream=None):
        check(lib().bg_cache_query(self.h, feat_dev, out_dev, int(n), _stream_handle(stream)))

    def train(self, feat_dev, target_dev, n, apply=True, want_loss=True, stream=None):
        loss = C.c_float()
        check(lib().bg_cache_train(self.h, feat_dev, target_dev, int(n), int(apply),
                                   C.byref(loss) if want_loss else None, _stream_handle(stream)))
        return loss.value if want_loss else None

    def params(self):
        inf = self.info()
        mlp = np.zeros(inf["mlp_params"], np.float32)
        grid = np.zeros(inf["grid_params"], np.float32)
        gm = np.zeros_like(mlp)
        gg = np.zeros_like(grid)
        check(lib().bg_cache_params(self.h, mlp.ctypes.data, grid.ctypes.data, gm.ctypes.data, gg.ctypes.data))
        return mlp, grid, gm, gg

    def set_params(self, mlp=None, grid=None):
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        check(lib().bg_cache_set_params(self.h, None if m is None else m.ctypes.data, None if g is None else g.ctypes.data))

    def render(self, accum_dev, width, height, spp, seed=1, sample_offset=0, maxdepth=8, camera=None, stream=None,
               flags=0, stats=False):
        sc = self.gs.scene
        cam = sc.camera_desc() if camera is None else camera
        tr = abi.TracerDesc(abi.BG_TRACER_GI, maxdepth, flags, 0)
        sm = abi.SamplerDesc(0, spp, seed, sample_offset, 0)
        st = abi.RenderStats()
        check(lib().bg_render_cached(self.gs.h, self.h, C.byref(cam), C.byref(tr), C.byref(sm), int(width), int(height),
                                     accum_dev, C.byref(st) if stats else None, _stream_handle(stream)))
        return {k: getattr(st, k) for k, _ in abi.RenderStats._fields_} if stats else None

    def close(self):
        if self.h:
            lib().bg_cache_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """bg_batch: several committed scenes rendered together from one set of queues."""

    def __init__(self, ctx, gscenes):
        self.ctx = ctx
        self.gscenes = list(gscenes)
        self.h = _vp()
        check(lib().bg_batch_create(ctx.h, C.byref(self.h)))
        for g in self.gscenes:
            check(lib().bg_batch_add_scene(self.h, g.h, None))
        check(lib().bg_batch_commit(self.h))

    def info(self):
        i = abi.SceneInfo()
        check(lib().bg_batch_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in abi.SceneInfo._fields_}

    def _jobs(self, jobs):
        arr = (abi.BatchJob * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            g = self.gscenes[j["scene"]]
            arr[i].scene = j["scene"]
            arr[i].width = j["width"]
            arr[i].height = j["height"]
            arr[i].camera = j.get("camera") or g.scene.camera_desc()
            arr[i].sampler = abi.SamplerDesc(j.get("sampler", 0), j["spp"], j.get("seed", 1),
                                             j.get("sample_offset", 0), j.get("grid", 0))
            arr[i].accum_rgbw_dev = j["accum_dev"]
        return arr

    def render(self, jobs, maxdepth=8, tracer=abi.BG_TRACER_GI, stream=None, stats=False, flags=0, ao_radius=0.0):
        arr = self._jobs(jobs)
        tr = abi.TracerDesc(tracer, maxdepth, flags, ao_radius)
        st = abi.RenderStats()
        check(lib().bg_batch_render(self.h, arr, len(jobs), C.byref(tr), C.byref(st) if stats else None,
                                    _stream_handle(stream)))
        return {k: getattr(st, k) for k, _ in abi.RenderStats._fields_} if stats else None

    def autotune(self, jobs, probe_spp=2, maxdepth=8, stream=None):
        arr = self._jobs(jobs)
        tr = abi.TracerDesc(abi.BG_TRACER_GI, maxdepth, 0, 0)
        res = abi.TuneResult()
        check(lib().bg_batch_autotune(self.h, arr, len(jobs), C.byref(tr), int(probe_spp), C.byref(res),
                                      _stream_handle(stream)))
        return {k: getattr(res, k) for k, _ in abi.TuneResult._fields_}

    def close(self):
        if self.h:
            lib().bg_batch_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def image_finalize(rgbw):
    """FileImagePlane::Finalize of a (H, W, 4) accumulation buffer -> (H, W, 3) floats."""
    a = np.ascontiguousarray(rgbw, dtype=np.float32)
    h, w = a.shape[0], a.shape[1]
    out = np.zeros((h, w, 3), np.float32)
    check(lib().bg_image_finalize(a.ctypes.data, w, h, out.ctypes.data))
    return out


def image_write(path, rgbw):
    """Write a (H, W, 4) accumulation buffer as .ppm (8-bit) or .pfm (float)."""
    a = np.ascontiguousarray(rgbw, dtype=np.float32)
    check(lib().bg_image_write(str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0]))
