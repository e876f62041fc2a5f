"""ctypes front-end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers with one interface:
  * ``Oracle``     -- the plain-C restatement (liboracle.so, banshee_oracle.c);
  * ``Reference``  -- Banshee's own sources compiled unmodified with the harness
                      in ref_harness.cpp (_ref/libbanshee_ref.so).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / CPU baseline.
"""
import ctypes as C
import os

import numpy as np

from banshee_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbanshee_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libbanshee_ref_gpu.so")

_vp = C.c_void_p


def _load_oracle():
    lib = C.CDLL(ORACLE_SO)
    lib.or_world_create.restype = _vp
    lib.or_world_create.argtypes = [_vp, C.c_int32, _vp, C.c_int32, _vp, C.c_int32, _vp]
    lib.or_world_destroy.argtypes = [_vp]
    lib.or_world_ntriangles.restype = C.c_int64
    lib.or_world_ntriangles.argtypes = [_vp]
    lib.or_world_nnodes.restype = C.c_int64
    lib.or_world_nnodes.argtypes = [_vp]
    lib.or_intersect_closest.argtypes = [_vp, _vp, _vp, C.c_int64, C.c_int32]
    lib.or_intersect_any.argtypes = [_vp, _vp, _vp, C.c_int64, C.c_int32]
    lib.or_traversal_counts.argtypes = [_vp, _vp, C.c_int64, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    lib.or_triangle_test.restype = C.c_int32
    lib.or_triangle_test.argtypes = [_vp, C.c_int64, _vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.or_render.argtypes = [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                              C.c_uint64, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                              C.c_int32, C.c_int32, C.c_float]
    lib.or_camera_rays.argtypes = [_vp, _vp, _vp, C.c_int64]
    lib.or_keyed_rand.restype = C.c_uint32
    lib.or_keyed_rand.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
    return lib


def _load_ref(path=REF_SO):
    lib = C.CDLL(path)
    lib.ref_world_create.restype = _vp
    lib.ref_world_create.argtypes = [_vp, C.c_int32, _vp, C.c_int32, _vp, C.c_int32, _vp, C.c_int32]
    lib.ref_world_destroy.argtypes = [_vp]
    lib.ref_intersect_closest.argtypes = [_vp, _vp, _vp, C.c_int64, C.c_int32]
    lib.ref_intersect_any.argtypes = [_vp, _vp, _vp, C.c_int64, C.c_int32]
    lib.ref_render.argtypes = [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                               C.c_uint64, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                               C.c_int32, C.c_int32, C.c_float]
    lib.ref_mcrng_draws.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int32, _vp]
    lib.ref_world_ntriangles.restype = C.c_int64
    lib.ref_world_ntriangles.argtypes = [_vp]
    return lib


_LIBS = {}


def _lib(kind):
    if kind not in _LIBS:
        if kind == "oracle":
            _LIBS[kind] = _load_oracle()
        elif kind == "ref_gpu":
            lib = _load_ref(REF_GPU_SO)
            lib.ref_world_use_gpu.restype = C.c_int32
            lib.ref_world_use_gpu.argtypes = [_vp, _vp]
            lib.ref_world_use_gpu_world.restype = C.c_int32
            lib.ref_world_use_gpu_world.argtypes = [_vp, _vp, C.POINTER(_vp)]
            lib.ref_gpu_renderer.restype = C.c_int32
            lib.ref_gpu_renderer.argtypes = [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_uint64, _vp]
            _LIBS[kind] = lib
        else:
            _LIBS[kind] = _load_ref()
    return _LIBS[kind]


def available(kind="oracle"):
    return os.path.exists({"oracle": ORACLE_SO, "ref_gpu": REF_GPU_SO}.get(kind, REF_SO))


def _addr(a):
    return a.ctypes.data


class _Checker:
    kind = None

    def __init__(self, scene, raycast=False):
        self.lib = _lib(self.kind)
        self._keep = scene.descs()
        marr, nm, mats, nmat, lights, nl, bg = self._keep
        self.scene = scene
        self.raycast = raycast
        self.w = self._create(marr, nm, mats, nmat, lights, nl, bg)
        if not self.w:
            raise ValueError("%s: world creation failed (invalid scene)" % self.kind)

    def close(self):
        if self.w:
            self._destroy(self.w)
            self.w = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def intersect_closest(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        hits = np.zeros(rays.shape[0], dtype=abi.HIT_DTYPE)
        self._closest(self.w, _addr(rays), _addr(hits), rays.shape[0], nthreads)
        return hits

    def intersect_any(self, rays, nthreads=0):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        occ = np.zeros(rays.shape[0], dtype=np.uint8)
        self._any(self.w, _addr(rays), _addr(occ), rays.shape[0], nthreads)
        return occ

    def render(self, camera=None, width=None, height=None, spp=1, seed=1, tracer=abi.BG_TRACER_GI,
               maxdepth=5, sample_offset=0, region=None, nthreads=0, accum=None, sampler=abi.BG_SAMPLER_RANDOM,
               grid=0, ao_radius=0.0):
        sc = self.scene
        width = width or sc.width
        height = height or sc.height
        cam = sc.camera_desc() if camera is None else camera
        if accum is None:
            accum = np.zeros((height, width, 4), dtype=np.float32)
        x0, y0, x1, y1 = region if region is not None else (0, 0, width, height)
        self._render(self.w, C.addressof(cam), tracer, maxdepth, width, height, spp, sample_offset, seed,
                     _addr(accum), x0, y0, x1, y1, nthreads, sampler, grid, ao_radius)
        return accum


class Oracle(_Checker):
    """The C restatement (banshee_oracle.c)."""
    kind = "oracle"

    def _create(self, marr, nm, mats, nmat, lights, nl, bg):
        return self.lib.or_world_create(C.addressof(marr), nm, C.addressof(mats), nmat,
                                        C.addressof(lights), nl, C.addressof(bg))

    def _destroy(self, w):
        self.lib.or_world_destroy(w)

    def _closest(self, *a):
        self.lib.or_intersect_closest(*a)

    def _any(self, *a):
        self.lib.or_intersect_any(*a)

    def _render(self, *a):
        self.lib.or_render(*a)

    def ntriangles(self):
        return self.lib.or_world_ntriangles(self.w)

    def traversal_counts(self, rays, any_hit=False):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        n, t = C.c_uint64(), C.c_uint64()
        self.lib.or_traversal_counts(self.w, _addr(rays), rays.shape[0], int(any_hit), C.byref(n), C.byref(t))
        return n.value, t.value

    def triangle_test(self, primid, ray):
        """Mesh::IntersectShape of one triangle; returns (t, u, v) or None."""
        r = np.ascontiguousarray(np.asarray(ray, dtype=abi.RAY_DTYPE).reshape(1))
        t, u, v = C.c_float(), C.c_float(), C.c_float()
        ok = self.lib.or_triangle_test(self.w, int(primid), _addr(r), C.byref(t), C.byref(u), C.byref(v))
        return (t.value, u.value, v.value) if ok else None

    def camera_rays(self, samples, camera=None):
        cam = self.scene.camera_desc() if camera is None else camera
        s = np.ascontiguousarray(samples, dtype=np.float32).reshape(-1, 2)
        rays = np.zeros(s.shape[0], dtype=abi.RAY_DTYPE)
        self.lib.or_camera_rays(C.addressof(cam), _addr(s), _addr(rays), s.shape[0])
        return rays


class Reference(_Checker):
    """Banshee's own sources (oracle/_ref), reached through its plugin surfaces."""
    kind = "ref"

    def _create(self, marr, nm, mats, nmat, lights, nl, bg):
        return self.lib.ref_world_create(C.addressof(marr), nm, C.addressof(mats), nmat,
                                         C.addressof(lights), nl, C.addressof(bg), int(self.raycast))

    def _destroy(self, w):
        self.lib.ref_world_destroy(w)

    def _closest(self, *a):
        if not self.raycast:
            raise ValueError("Reference ray casts need raycast=True (primitive ids come from Hit::m)")
        self.lib.ref_intersect_closest(*a)

    def _any(self, *a):
        self.lib.ref_intersect_any(*a)

    def _render(self, *a):
        if self.raycast:
            raise ValueError("render needs a world built with raycast=False")
        self.lib.ref_render(*a)


def keyed_rand(seed, pixel, sample, counter):
    return _lib("oracle").or_keyed_rand(seed, pixel, sample, counter)


def ref_mcrng_draws(seed, pixel, sample, n):
    out = np.zeros((n, 2), dtype=np.float32)
    _lib("ref").ref_mcrng_draws(seed, pixel, sample, n, _addr(out))
    return out


class ReferenceOnGpu(Reference):
    """Banshee's own sources whose World answers Intersect through the
    GpuAccelerator adapter once use_gpu() is called (before: its own Bvh)."""
    kind = "ref_gpu"

    def gpu_renderer(self, gpu_scene_handle, spp, frames, seed=1, tracer=abi.BG_TRACER_GI, maxdepth=5):
        """GpuRenderer::Render called `frames` times (spp samples each) on this world."""
        sc = self.scene
        cam = sc.camera_desc()
        accum = np.zeros((sc.height, sc.width, 4), dtype=np.float32)
        if self.lib.ref_gpu_renderer(self.w, gpu_scene_handle, C.addressof(cam), tracer, maxdepth, sc.width,
                                     sc.height, spp, frames, seed, _addr(accum)) != 0:
            raise ValueError("GpuRenderer failed")
        return accum

    def use_gpu(self, gpu_scene_handle):
        if self.lib.ref_world_use_gpu(self.w, gpu_scene_handle) != 0:
            raise ValueError("GpuAccelerator rejected the world")

    def use_gpu_world(self, gpu_ctx_handle):
        """GpuAccelerator over a device scene built from this committed World
        (gpu_scene_from_world); returns the scene handle, which the caller
        destroys (bg_scene_destroy) after close()."""
        h = _vp()
        if self.lib.ref_world_use_gpu_world(self.w, gpu_ctx_handle, C.byref(h)) != 0:
            raise ValueError("gpu_scene_from_world or GpuAccelerator failed")
        return h.value
