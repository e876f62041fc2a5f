"""ctypes mirror of the C ABI structs declared in include/banshee_gpu.h.

Ray and hit arrays are numpy structured arrays with the exact byte layout of
``bg_ray`` (32 B) and ``bg_hit`` (16 B), so they can be handed to the library
(or copied to the device) without repacking.
"""
import ctypes as C

import numpy as np

BG_OK = 0
BG_ERR = {
    -1: "BG_ERR_INVALID_ARG", -2: "BG_ERR_CUDA", -3: "BG_ERR_OOM", -4: "BG_ERR_STATE",
    -5: "BG_ERR_OVERFLOW", -6: "BG_ERR_TIMEOUT", -7: "BG_ERR_UNSUPPORTED", -8: "BG_ERR_NO_DEVICE",
}

BG_MAT_LAMBERT, BG_MAT_MICROFACET_GGX, BG_MAT_EMISSIVE = 0, 1, 2
BG_LIGHT_AREA, BG_LIGHT_DIRECTIONAL, BG_LIGHT_ENVIRONMENT = 0, 1, 2
BG_TRACER_GI, BG_TRACER_DI, BG_TRACER_AO = 0, 1, 2

RAY_DTYPE = np.dtype([("o", "<f4", 3), ("tmin", "<f4"), ("d", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("primid", "<i4"), ("u", "<f4"), ("v", "<f4")])
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [
        ("vertices", _fp), ("nvertices", C.c_int32), ("vstride", C.c_int32),
        ("normals", _fp), ("nnormals", C.c_int32), ("nstride", C.c_int32),
        ("uvs", _fp), ("nuvs", C.c_int32), ("ustride", C.c_int32),
        ("vidx", _ip), ("vistride", C.c_int32),
        ("nidx", _ip), ("nistride", C.c_int32),
        ("uidx", _ip), ("uistride", C.c_int32),
        ("materials", _ip), ("mstride", C.c_int32),
        ("nfaces", C.c_int32),
        ("m", C.c_float * 16), ("minv", C.c_float * 16),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("kd", C.c_float * 3), ("ks", C.c_float * 3),
                ("eta", C.c_float), ("roughness", C.c_float), ("e", C.c_float * 3)]


class LightDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("mesh", C.c_int32), ("face", C.c_int32),
                ("d", C.c_float * 3), ("e", C.c_float * 3), ("scale", C.c_float), ("gamma", C.c_float)]


class CameraDesc(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("at", C.c_float * 3), ("up", C.c_float * 3),
                ("znear", C.c_float), ("zfar", C.c_float), ("fovy", C.c_float), ("aspect", C.c_float)]


class BuildOpts(C.Structure):
    _fields_ = [("node_width", C.c_int32), ("max_leaf_size", C.c_int32),
                ("sah_bins", C.c_int32), ("builder", C.c_int32), ("intersect", C.c_int32)]


BG_INTERSECT_REFERENCE, BG_INTERSECT_WATERTIGHT = 0, 1


class SceneInfo(C.Structure):
    _fields_ = [("ntriangles", C.c_int64), ("nnodes", C.c_int64), ("node_bytes", C.c_int64),
                ("tri_bytes", C.c_int64), ("shade_bytes", C.c_int64), ("node_stride", C.c_int32),
                ("max_depth", C.c_int32), ("max_stack", C.c_int32), ("nmeshes", C.c_int32),
                ("nmaterials", C.c_int32), ("nlights", C.c_int32), ("build_ms", C.c_double),
                ("node_width", C.c_int32), ("node_widths", C.c_int32), ("bvh_ms", C.c_double),
                ("records_ms", C.c_double), ("upload_ms", C.c_double)]


BG_SAMPLER_RANDOM, BG_SAMPLER_SOBOL, BG_SAMPLER_CMJ = 0, 1, 2

BG_RENDER_TIME_PHASES = 0x1
BG_RENDER_COUNT_TRAVERSAL = 0x2


class TracerDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("maxdepth", C.c_int32), ("flags", C.c_int32), ("ao_radius", C.c_float)]


class SamplerDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("spp", C.c_int32), ("seed", C.c_uint64),
                ("sample_offset", C.c_int32), ("grid", C.c_int32)]


class RenderStats(C.Structure):
    _fields_ = [("camera_samples", C.c_int64), ("rays_extension", C.c_int64), ("rays_closest", C.c_int64),
                ("rays_any", C.c_int64), ("kernel_launches", C.c_int64),
                ("ms_total", C.c_float), ("ms_extend", C.c_float), ("ms_mis", C.c_float), ("ms_shadow", C.c_float),
                ("ms_shade", C.c_float), ("launches_extend", C.c_int32),
                ("ms_cache_query", C.c_float), ("ms_cache_train", C.c_float),
                ("sub_rays_extension", C.c_int64), ("sub_nodes_extension", C.c_int64),
                ("sub_tris_extension", C.c_int64),
                ("sub_rays_any", C.c_int64), ("sub_nodes_any", C.c_int64), ("sub_tris_any", C.c_int64),
                ("sub_rays_mis", C.c_int64), ("sub_nodes_mis", C.c_int64), ("sub_tris_mis", C.c_int64)]


class CacheDesc(C.Structure):
    _fields_ = [("levels", C.c_int32), ("log2_table_size", C.c_int32), ("base_resolution", C.c_int32),
                ("max_resolution", C.c_int32), ("train_paths", C.c_int32), ("cache_depth", C.c_int32),
                ("train_batch", C.c_int32), ("train_steps", C.c_int32), ("learning_rate", C.c_float),
                ("bbox_min", C.c_float * 3), ("bbox_max", C.c_float * 3), ("seed", C.c_uint64),
                ("mlp_kernel", C.c_int32), ("train_suffix", C.c_int32), ("wait_polls", C.c_int32)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("reserved", C.c_int32),
                ("camera", CameraDesc), ("sampler", SamplerDesc), ("accum_rgbw_dev", C.c_void_p)]


class TuneResult(C.Structure):
    _fields_ = [("trace_threads", C.c_int32), ("paths_per_pass", C.c_int32), ("candidates", C.c_int32),
                ("ms", C.c_float), ("msamples_per_s", C.c_float), ("node_width", C.c_int32)]


def fptr(a):
    return a.ctypes.data_as(_fp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


class AllocStats(C.Structure):
    _fields_ = [("calls", C.c_int64), ("bytes", C.c_int64), ("refused", C.c_int64), ("budget", C.c_int64)]
