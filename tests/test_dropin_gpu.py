"""The drop-in itself: Banshee's own World, tracers, samplers and renderer
(the reference sources compiled unmodified) with World::accel_ replaced by the
GpuAccelerator adapter over the C ABI.  Every closest hit and every shadow
query of the reference's GiTracer / DiTracer then comes from the GPU, and the
images must be bit-identical to the same code running on its own Bvh."""
import ctypes as C
import os

import numpy as np
import pytest

from banshee_b200 import abi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


@pytest.fixture(scope="module")
def ref_gpu():
    from oracle import oracle
    if not oracle.available("ref_gpu"):
        pytest.skip("oracle/_ref/libbanshee_ref_gpu.so not built (needs the reference tree at build time)")
    return oracle


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("tracer", [abi.BG_TRACER_GI, abi.BG_TRACER_DI])
def test_reference_tracer_over_gpu_accelerator(ctx, ref_gpu, tracer, width):
    from banshee_b200 import capi
    sc = scenes.cornell(24, 24)
    gs = capi.GpuScene(ctx, sc)
    gs.set_node_width(width)
    ref = ref_gpu.ReferenceOnGpu(sc)
    kw = dict(spp=4, seed=9, tracer=tracer, maxdepth=5, nthreads=4)
    own = ref.render(**kw)                 # the reference's Bvh
    ref.use_gpu(gs.h.value)
    gpu = ref.render(**kw)                 # the same reference code, hits from the GPU
    assert (own.view(np.uint32) == gpu.view(np.uint32)).all()
    assert gs.error_flags() == 0


@pytest.mark.parametrize("scene", ["cornell", "production"])
def test_gpu_accelerator_over_scene_built_from_the_world(ctx, ref_gpu, scene):
    """gpu_scene_from_world builds the device scene from the committed World's
    own bundles (vertices, faces, transforms through public accessors), with no
    scene description from the caller; the reference's tracer over it renders
    the same image, bit for bit, as over its own Bvh."""
    from banshee_b200 import capi
    if scene == "cornell":
        sc = scenes.cornell(20, 20)
        kw = dict(spp=4, seed=9, tracer=abi.BG_TRACER_GI, maxdepth=5, nthreads=4)
    else:   # transformed bundles
        sc = scenes.production(20, 12, nterrain=32, nspheres=6, sphere_seg=10, seed=4)
        kw = dict(spp=2, seed=3, maxdepth=8, nthreads=4)
    ref = ref_gpu.ReferenceOnGpu(sc)
    own = ref.render(**kw)
    handle = ref.use_gpu_world(ctx.h.value)
    try:
        gpu = ref.render(**kw)
        assert (own.view(np.uint32) == gpu.view(np.uint32)).all()
        flags = C.c_uint32()
        assert capi.lib().bg_scene_error_flags(C.c_void_p(handle), C.byref(flags), 1) == 0 and flags.value == 0
    finally:
        ref.close()
        capi.lib().bg_scene_destroy(C.c_void_p(handle))


def test_reference_production_scene_over_gpu_accelerator(ctx, ref_gpu):
    """Transformed bundles (spheres), GGX, sun and environment."""
    from banshee_b200 import capi
    sc = scenes.production(24, 14, nterrain=32, nspheres=6, sphere_seg=10, seed=4)
    gs = capi.GpuScene(ctx, sc)
    ref = ref_gpu.ReferenceOnGpu(sc)
    kw = dict(spp=2, seed=3, maxdepth=8, nthreads=4)
    own = ref.render(**kw)
    ref.use_gpu(gs.h.value)
    gpu = ref.render(**kw)
    assert (own.view(np.uint32) == gpu.view(np.uint32)).all()


def test_gpu_renderer_adapter_matches_reference_renderer(ctx, ref_gpu):
    """Renderer::Render through the GpuRenderer adapter, 3 progressive frames of
    4 samples, against the reference's own renderer with the same 12 samples."""
    from banshee_b200 import capi
    from banshee_b200.metrics import mean_image, relmse
    sc = scenes.cornell(32, 32)
    gs = capi.GpuScene(ctx, sc)
    ref = ref_gpu.ReferenceOnGpu(sc)
    got = ref.gpu_renderer(gs.h.value, spp=4, frames=3, seed=5, maxdepth=5)
    want = ref.render(spp=12, seed=5, maxdepth=5, nthreads=4)
    assert (got[..., 3] == want[..., 3]).all()
    assert relmse(mean_image(got), mean_image(want)) < 1e-4


def test_concurrent_host_casts_run_side_by_side(ctx, ref_gpu):
    """GpuAccelerator is called one ray at a time from every renderer thread.
    Each thread casts through its own staging (stream, buffers, work counter),
    so more threads give more rays per second, and the image stays identical."""
    import time
    from banshee_b200 import capi
    sc = scenes.cornell(32, 32)
    gs = capi.GpuScene(ctx, sc)
    ref = ref_gpu.ReferenceOnGpu(sc)
    own = ref.render(spp=2, seed=4, maxdepth=5, nthreads=8)
    ref.use_gpu(gs.h.value)
    rate = {}
    for nt in (1, 8):
        t0 = time.perf_counter()
        img = ref.render(spp=2, seed=4, maxdepth=5, nthreads=nt)
        rate[nt] = 32 * 32 * 2 / (time.perf_counter() - t0)
        assert (img.view(np.uint32) == own.view(np.uint32)).all()
    print("reference GiTracer over GpuAccelerator: %.0f samples/s on 1 thread, %.0f on 8" % (rate[1], rate[8]))
    assert rate[8] > 2.0 * rate[1], rate
    assert gs.error_flags() == 0
