"""Multi-scene batches: scenes of uneven size, resolution and spp traced
together from one set of queues.  Each job's image must be bit-identical to
rendering its scene alone (same geometry, same traversal order, same sampler
sequences, same per-pixel summation order), including after autotuning."""
import numpy as np
import pytest

from banshee_b200 import abi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


def _scenes():
    return [
        (scenes.cornell(40, 40), 5, 5),
        (scenes.production(64, 36, nterrain=32, nspheres=6, sphere_seg=10, seed=11), 3, 8),
        (scenes.production(48, 48, nterrain=40, nspheres=3, sphere_seg=8, seed=12), 7, 8),
        (scenes.cornell(24, 16), 2, 5),
    ]


@pytest.mark.parametrize("tune", [False, True])
def test_batch_jobs_match_single_scene_renders(ctx, tune):
    import torch
    from banshee_b200 import capi
    items = _scenes()
    gss = [capi.GpuScene(ctx, sc) for sc, _, _ in items]
    batch = capi.Batch(ctx, gss)
    info = batch.info()
    assert info["ntriangles"] == sum(sc.ntriangles for sc, _, _ in items)
    # two jobs per scene (different seeds), one maxdepth for the whole batch
    maxdepth = 5
    jobs, bufs = [], []
    for k, (sc, spp, _) in enumerate(items):
        for seed in (1, 2):
            acc = torch.zeros((sc.height, sc.width, 4), dtype=torch.float32, device="cuda")
            bufs.append(acc)
            jobs.append(dict(scene=k, width=sc.width, height=sc.height, spp=spp, seed=seed, accum_dev=acc.data_ptr()))
    if tune:
        res = batch.autotune(jobs, probe_spp=1, maxdepth=maxdepth)
        probe = sum(j["width"] * j["height"] for j in jobs)
        # node widths x block sizes x the pass sizes 2^19.. that the probe does not fit in half of
        npass = 1 + sum(1 for i in range(1, 6) if (1 << (19 + i)) // 2 < probe)
        assert res["candidates"] == 2 * 2 * npass
        assert res["trace_threads"] in (128, 256) and res["node_width"] in (4, 8)
        assert batch.info()["node_width"] == res["node_width"]
        for b in bufs:
            b.zero_()
    batch.render(jobs, maxdepth=maxdepth)
    torch.cuda.synchronize()
    for j, acc in zip(jobs, bufs):
        sc, spp, _ = items[j["scene"]]
        ref = gss[j["scene"]].render_host(sc.width, sc.height, spp, seed=j["seed"], maxdepth=maxdepth)
        got = acc.cpu().numpy()
        assert (got.view(np.uint32) == ref.view(np.uint32)).all(), (j["scene"], j["seed"])


def test_batch_progressive_and_stats(ctx):
    import torch
    from banshee_b200 import capi
    items = _scenes()[:2]
    gss = [capi.GpuScene(ctx, sc) for sc, _, _ in items]
    batch = capi.Batch(ctx, gss)
    bufs = [torch.zeros((sc.height, sc.width, 4), dtype=torch.float32, device="cuda") for sc, _, _ in items]
    for off in (0, 3):
        jobs = [dict(scene=k, width=sc.width, height=sc.height, spp=3, seed=4, sample_offset=off,
                     accum_dev=bufs[k].data_ptr()) for k, (sc, _, _) in enumerate(items)]
        st = batch.render(jobs, maxdepth=5, stats=True)
    assert st["camera_samples"] == sum(sc.width * sc.height * 3 for sc, _, _ in items)
    torch.cuda.synchronize()
    for k, (sc, _, _) in enumerate(items):
        ref = gss[k].render_host(sc.width, sc.height, 6, seed=4, maxdepth=5)
        assert (bufs[k].cpu().numpy().view(np.uint32) == ref.view(np.uint32)).all()
