"""Wavefront GI / DI tracer parity on the GPU.

With the same keyed sampler sequences, GPU images must match Banshee's own
CPU tracer (golden fixtures from the reference, and the CPU restatement at
larger sizes) within relMSE 1e-4 (mean over pixels and channels of
(x - ref)^2 / (ref^2 + 0.01)).  The only arithmetic difference is CUDA's
sinf/cosf/powf/atanf versus libm's (a few ulp)."""
import os

import numpy as np
import pytest

from banshee_b200 import abi, scenes
from banshee_b200.metrics import mean_image, relmse

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


def _render(ctx, sc, spp, seed, tracer, maxdepth, width=4, **kw):
    from banshee_b200 import capi
    gs = capi.GpuScene(ctx, sc)
    gs.set_node_width(width)
    img = gs.render_host(sc.width, sc.height, spp, seed=seed, tracer=tracer, maxdepth=maxdepth, **kw)
    assert gs.error_flags() == 0
    return img


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("tracer", ["gi", "di"])
def test_cornell_matches_reference_golden(ctx, tracer, width):
    from tests.golden.make_golden import CORNELL
    g = np.load(os.path.join(GOLD, "render_cornell.npz"))
    kind = abi.BG_TRACER_GI if tracer == "gi" else abi.BG_TRACER_DI
    img = _render(ctx, scenes.cornell(**CORNELL), int(g["spp"]), int(g["seed"]), kind, int(g["maxdepth"]),
                  width=width)
    ref = g[tracer]
    assert (img[..., 3] == ref[..., 3]).all()          # sample counts
    e = relmse(mean_image(img), mean_image(ref))
    assert e < TOL, e


@pytest.mark.parametrize("width", [4, 8])
def test_production_ggx_matches_reference_golden(ctx, width):
    from tests.golden.make_golden import PROD
    g = np.load(os.path.join(GOLD, "render_production.npz"))
    img = _render(ctx, scenes.production(**PROD), int(g["spp"]), int(g["seed"]), abi.BG_TRACER_GI, int(g["maxdepth"]),
                  width=width)
    e = relmse(mean_image(img), mean_image(g["gi"]))
    assert e < TOL, e


@pytest.mark.parametrize("maxdepth", [5, 8])
def test_cornell_vs_oracle_larger(ctx, oracle_built, maxdepth):
    sc = scenes.cornell(96, 96)
    img = _render(ctx, sc, 16, 3, abi.BG_TRACER_GI, maxdepth)
    ref = oracle_built.Oracle(sc).render(spp=16, seed=3, maxdepth=maxdepth)
    e = relmse(mean_image(img), mean_image(ref))
    assert e < TOL, e


@pytest.mark.parametrize("width", [4, 8])
def test_production_vs_oracle_larger(ctx, oracle_built, width):
    sc = scenes.production(160, 90, nterrain=96, nspheres=24, sphere_seg=16, seed=5)
    img = _render(ctx, sc, 4, 4, abi.BG_TRACER_GI, 8, width=width)
    ref = oracle_built.Oracle(sc).render(spp=4, seed=4, maxdepth=8)
    e = relmse(mean_image(img), mean_image(ref))
    assert e < TOL, e


def test_deterministic_and_progressive(ctx):
    from banshee_b200 import capi
    sc = scenes.cornell(48, 48)
    gs = capi.GpuScene(ctx, sc)
    a = gs.render_host(48, 48, 6, seed=9)
    b = gs.render_host(48, 48, 6, seed=9)
    assert (a.view(np.uint32) == b.view(np.uint32)).all()
    c = gs.render_host(48, 48, 2, seed=9)
    c = gs.render_host(48, 48, 4, seed=9, sample_offset=2, accum=c)
    assert (a.view(np.uint32) == c.view(np.uint32)).all()
    assert (a[..., 3] == 6).all()


def test_graph_replay_matches_direct_launches(ctx):
    """Without statistics a pass is replayed from a captured CUDA graph; with
    statistics its kernels are launched one by one: same bits either way."""
    import torch
    from banshee_b200 import capi
    sc = scenes.production(96, 54, nterrain=48, nspheres=12, sphere_seg=12, seed=3)
    gs = capi.GpuScene(ctx, sc)
    a = torch.zeros((54, 96, 4), dtype=torch.float32, device="cuda")
    b = torch.zeros_like(a)
    for k in range(3):     # repeated replays with changing sample offsets
        gs.render(a.data_ptr(), 96, 54, 2, seed=4, sample_offset=2 * k, maxdepth=8, stats=False)
        gs.render(b.data_ptr(), 96, 54, 2, seed=4, sample_offset=2 * k, maxdepth=8, stats=True)
    torch.cuda.synchronize()
    assert (a.cpu().numpy().view(np.uint32) == b.cpu().numpy().view(np.uint32)).all()
    assert gs.error_flags() == 0


@pytest.mark.parametrize("kind", [abi.BG_TRACER_GI, abi.BG_TRACER_DI, abi.BG_TRACER_AO])
def test_late_direct_light_matches_serial_order(ctx, kind):
    """An uninstrumented pass resolves direct light one bounce late on a side
    stream (slot halves by bounce parity); phase timing runs the bounces in
    serial order.  Every tracer kind gives the same bits both ways, on a
    scene with area lights (MIS rays) and on the sun + environment scene."""
    import torch
    from banshee_b200 import capi
    for sc in (scenes.cornell(40, 40),
               scenes.production(64, 36, nterrain=32, nspheres=6, sphere_seg=10, seed=7)):
        gs = capi.GpuScene(ctx, sc)
        W, H = sc.width, sc.height
        kw = dict(tracer=kind, maxdepth=1 if kind == abi.BG_TRACER_AO else 8,
                  ao_radius=0.5 if kind == abi.BG_TRACER_AO else 0.0)
        late = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        serial = torch.zeros_like(late)
        gs.render(late.data_ptr(), W, H, 3, seed=11, stats=False, **kw)
        st = gs.render(serial.data_ptr(), W, H, 3, seed=11, stats=True, flags=abi.BG_RENDER_TIME_PHASES, **kw)
        torch.cuda.synchronize()
        assert st["camera_samples"] == W * H * 3
        assert (late.cpu().numpy().view(np.uint32) == serial.cpu().numpy().view(np.uint32)).all(), sc.name
        assert gs.error_flags() == 0
        gs.close()


@pytest.mark.parametrize("flags", [0, 1, 3])
def test_host_entry_overlapped_upload_then_every_launch_path(ctx, flags):
    """bg_render_host uploads the accumulation buffer on a copy stream that
    only the pass's accumulate waits for.  Progressive host frames, then device
    renders replayed from the graph, launched one by one (statistics) and
    instrumented (phase timing / traversal counting), all give the bits of one
    direct render of the same samples."""
    import torch
    from banshee_b200 import capi
    sc = scenes.production(96, 54, nterrain=48, nspheres=12, sphere_seg=12, seed=5)
    gs = capi.GpuScene(ctx, sc)
    host = np.zeros((54, 96, 4), dtype=np.float32)
    for k in range(3):
        host = gs.render_host(96, 54, 1, seed=6, sample_offset=k, maxdepth=8, accum=host)
    dev = torch.zeros((54, 96, 4), dtype=torch.float32, device="cuda")
    for k in range(3):
        gs.render(dev.data_ptr(), 96, 54, 1, seed=6, sample_offset=k, maxdepth=8, stats=(k == 1), flags=flags)
    one = torch.zeros_like(dev)
    gs.render(one.data_ptr(), 96, 54, 3, seed=6, maxdepth=8, stats=False)
    torch.cuda.synchronize()
    want = one.cpu().numpy().view(np.uint32)
    assert (dev.cpu().numpy().view(np.uint32) == want).all()
    assert (host.view(np.uint32) == want).all()
    assert gs.error_flags() == 0


def test_device_render_entry_point(ctx):
    import torch
    from banshee_b200 import capi
    sc = scenes.cornell(64, 64)
    gs = capi.GpuScene(ctx, sc)
    acc = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
    st = gs.render(acc.data_ptr(), 64, 64, 4, seed=2)
    assert st["camera_samples"] == 64 * 64 * 4
    assert st["rays_closest"] >= 64 * 64 * 4 and st["rays_any"] > 0
    host = gs.render_host(64, 64, 4, seed=2)
    assert (acc.cpu().numpy().view(np.uint32) == host.view(np.uint32)).all()


def test_render_argument_errors(ctx):
    from banshee_b200 import capi
    sc = scenes.cornell(8, 8)
    gs = capi.GpuScene(ctx, sc)
    with pytest.raises(capi.BansheeError):
        gs.render_host(0, 8, 1)
    with pytest.raises(capi.BansheeError):
        gs.render_host(8, 8, 1, tracer=7)


SAMPLER_CASES = [
    ("gi_sobol", dict(tracer=abi.BG_TRACER_GI, maxdepth=5, sampler=abi.BG_SAMPLER_SOBOL)),
    ("gi_cmj4", dict(tracer=abi.BG_TRACER_GI, maxdepth=5, sampler=abi.BG_SAMPLER_CMJ, grid=4, sample_offset=3)),
    ("ao", dict(tracer=abi.BG_TRACER_AO, maxdepth=1, ao_radius=0.25)),
    ("ao_sobol", dict(tracer=abi.BG_TRACER_AO, maxdepth=1, ao_radius=0.25, sampler=abi.BG_SAMPLER_SOBOL)),
]


@pytest.mark.parametrize("name,kw", SAMPLER_CASES, ids=[c[0] for c in SAMPLER_CASES])
def test_samplers_and_ao_match_reference_golden(ctx, name, kw):
    """Sobol / CMJ image samplers and AoTracer against the reference's own
    SobolSampler, CmjSampler and AoTracer."""
    from tests.golden.make_golden import CORNELL
    g = np.load(os.path.join(GOLD, "render_samplers.npz"))
    kw = dict(kw)
    img = _render(ctx, scenes.cornell(**CORNELL), int(g["spp"]), int(g["seed"]), kw.pop("tracer"), kw.pop("maxdepth"),
                  **kw)
    ref = g[name]
    assert (img[..., 3] == ref[..., 3]).all()
    e = relmse(mean_image(img), mean_image(ref))
    assert e < TOL, e


def test_ao_and_samplers_vs_oracle_production(ctx, oracle_built):
    sc = scenes.production(120, 68, nterrain=64, nspheres=16, sphere_seg=12, seed=6)
    o = oracle_built.Oracle(sc)
    for kw in (dict(tracer=abi.BG_TRACER_AO, maxdepth=1, ao_radius=2.0, sampler=abi.BG_SAMPLER_CMJ, grid=2),
               dict(tracer=abi.BG_TRACER_GI, maxdepth=8, sampler=abi.BG_SAMPLER_SOBOL, sample_offset=11)):
        img = _render(ctx, sc, 4, 5, **kw)
        ref = o.render(spp=4, seed=5, **kw)
        e = relmse(mean_image(img), mean_image(ref))
        assert e < TOL, (kw, e)


def test_node_layouts_give_identical_images(ctx):
    """Both node layouts return the same closest hits, so whole images agree bit for bit."""
    from banshee_b200 import capi
    sc = scenes.production(96, 54, nterrain=64, nspheres=16, sphere_seg=12, seed=8)
    gs = capi.GpuScene(ctx, sc)
    imgs = []
    for w in (4, 8):
        gs.set_node_width(w)
        imgs.append(gs.render_host(96, 54, 8, seed=2, maxdepth=8))
    assert (imgs[0].view(np.uint32) == imgs[1].view(np.uint32)).all()
    assert gs.error_flags() == 0


def test_scene_autotune_keeps_images_bit_identical(ctx):
    """bg_scene_autotune only changes node layout, block size and pass size:
    renders before and after it agree bit for bit."""
    import torch
    from banshee_b200 import capi
    sc = scenes.production(80, 45, nterrain=48, nspheres=8, sphere_seg=10, seed=2)
    gs = capi.GpuScene(ctx, sc)
    before = gs.render_host(80, 45, 6, seed=4, maxdepth=8)
    probe = torch.zeros((45, 80, 4), dtype=torch.float32, device="cuda")
    res = gs.autotune(probe.data_ptr(), 80, 45, probe_spp=1, maxdepth=8)
    torch.cuda.synchronize()
    # node widths x block sizes x one pass size: 3,600 probe samples fit in 2^19 / 2
    assert res["candidates"] == 4 and res["node_width"] in (4, 8) and res["trace_threads"] in (128, 256)
    assert gs.info()["node_width"] == res["node_width"]
    assert (probe.cpu().numpy()[..., 3] == 8).all()        # 4 candidates x 2 probe renders x 1 spp
    after = gs.render_host(80, 45, 6, seed=4, maxdepth=8)
    assert (before.view(np.uint32) == after.view(np.uint32)).all()
