"""Neural radiance cache on the GPU.

* gradients of the MLP weights and of the hash grid from the project's own
  backward kernels match the float64 CPU oracle (oracle/nrc_oracle.py, which
  emulates bf16 rounding at the same points) -- cosine > 0.999 and relative
  L2 error < 2e-2 per parameter block;
* the forward pass (bg_cache_query) matches the oracle;
* Adam training on a smooth synthetic radiance field lowers the loss;
* the cache-mode tracer renders finite images and trains online;
* what the trained network gains: on the Cornell box (long, bright indirect
  paths), ending paths after 2 bounces without a cache (plain tracer at max
  depth 2) misses the light carried by longer paths; ending them into the
  online-trained cache recovers it, so the error against a deep reference
  render falls several-fold at the same cost structure.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


def _features(n, rng, bbox=((0, 0, 0), (1, 1, 1))):
    lo, hi = np.array(bbox[0], np.float32), np.array(bbox[1], np.float32)
    f = np.zeros((n, 16), np.float32)
    f[:, 0:3] = lo + rng.random((n, 3)).astype(np.float32) * (hi - lo)
    d = rng.normal(size=(n, 3))
    f[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    m = rng.normal(size=(n, 3))
    f[:, 6:9] = m / np.linalg.norm(m, axis=1, keepdims=True)
    f[:, 9] = rng.random(n)
    f[:, 10:13] = rng.random((n, 3))
    return f


def _cache(ctx, log2t=8, **kw):
    from banshee_b200 import capi, scenes
    gs = capi.GpuScene(ctx, scenes.cornell(8, 8))
    return gs, capi.RadianceCache(gs, log2_table_size=log2t, base_resolution=4, max_resolution=64,
                                  bbox=((0, 0, 0), (1, 1, 1)), **kw)


def _oracle_args(cache):
    inf = cache.info()
    return inf["resolutions"], cache.log2_table_size, inf["bmin"], inf["bscale"]


@pytest.mark.parametrize("mlp_kernel", [0, 1], ids=["tcgen05", "mma_sync"])
def test_gradients_match_fp64_oracle(ctx, mlp_kernel):
    import torch
    from oracle import nrc_oracle as O
    gs, cache = _cache(ctx, log2t=8, mlp_kernel=mlp_kernel)
    rng = np.random.default_rng(3)
    mlp0, grid0, _, _ = cache.params()
    # non-trivial grid values so that the grid features matter
    grid = (rng.random(grid0.shape).astype(np.float32) - 0.5) * 0.5
    cache.set_params(mlp0, grid)
    n = 777
    feat = _features(n, rng)
    target = np.zeros((n, 4), np.float32)
    target[:, :3] = rng.random((n, 3)) * 2
    fd = torch.from_numpy(feat).cuda()
    td = torch.from_numpy(target).cuda()
    loss = cache.train(fd.data_ptr(), td.data_ptr(), n, apply=False)
    mlp, g, dmlp, dgrid = cache.params()
    res, log2t, bmin, bscale = _oracle_args(cache)
    ref_loss, ref_dmlp, ref_dgrid, _ = O.loss_and_grads(feat.astype(np.float64), target.astype(np.float64), mlp, g,
                                                        res, log2t, bmin, bscale)
    assert abs(loss - ref_loss) <= 1e-2 * abs(ref_loss) + 1e-6, (loss, ref_loss)
    for k in range(6):
        a = dmlp[O.W_OFFS[k]:O.W_OFFS[k + 1]].astype(np.float64)
        b = ref_dmlp[O.W_OFFS[k]:O.W_OFFS[k + 1]]
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
        assert cos > 0.999 and rel < 2e-2, (k, cos, rel)
    a, b = dgrid.astype(np.float64), ref_dgrid
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
    assert cos > 0.999 and np.linalg.norm(a - b) / np.linalg.norm(b) < 2e-2, cos


@pytest.mark.parametrize("mlp_kernel", [0, 1], ids=["tcgen05", "mma_sync"])
def test_forward_matches_oracle(ctx, mlp_kernel):
    import torch
    from oracle import nrc_oracle as O
    gs, cache = _cache(ctx, log2t=10, mlp_kernel=mlp_kernel)
    rng = np.random.default_rng(5)
    n = 1000
    feat = _features(n, rng)
    fd = torch.from_numpy(feat).cuda()
    out = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    cache.query(fd.data_ptr(), out.data_ptr(), n)
    torch.cuda.synchronize()
    mlp, g, _, _ = cache.params()
    res, log2t, bmin, bscale = _oracle_args(cache)
    X, _ = O.encode(feat.astype(np.float64), g, res, log2t, bmin, bscale)
    ref, _, _ = O.forward(X, mlp)
    got = out.cpu().numpy()[:, :3]
    err = np.abs(got - ref[:, :3]).max() / (np.abs(ref[:, :3]).max() + 1e-12)
    assert err < 2e-2, err


@pytest.mark.parametrize("mlp_kernel", [0, 1], ids=["tcgen05", "mma_sync"])
def test_adam_training_reduces_loss(ctx, mlp_kernel):
    import torch
    gs, cache = _cache(ctx, log2t=12, learning_rate=1e-2, mlp_kernel=mlp_kernel)
    rng = np.random.default_rng(7)
    n = 16384
    feat = _features(n, rng)
    p = feat[:, 0:3]
    target = np.zeros((n, 4), np.float32)
    target[:, 0] = 0.5 + 0.4 * np.sin(6 * p[:, 0]) * np.cos(4 * p[:, 1])
    target[:, 1] = 0.3 + 0.2 * p[:, 2] + 0.1 * feat[:, 5]
    target[:, 2] = 0.2 + 0.2 * feat[:, 10]
    fd = torch.from_numpy(feat).cuda()
    td = torch.from_numpy(target).cuda()
    first = cache.train(fd.data_ptr(), td.data_ptr(), n, apply=True)
    for _ in range(300):
        last = cache.train(fd.data_ptr(), td.data_ptr(), n, apply=True, want_loss=False)
    last = cache.train(fd.data_ptr(), td.data_ptr(), n, apply=False)
    assert np.isfinite(last) and last < 0.1 * first, (first, last)


def test_cached_render_trains_online(ctx):
    import torch
    from banshee_b200 import capi, scenes
    sc = scenes.production(96, 54, nterrain=48, nspheres=12, sphere_seg=12, seed=3)
    gs = capi.GpuScene(ctx, sc)
    cache = capi.RadianceCache(gs, log2_table_size=14, train_paths=2048, train_batch=4096, train_steps=2)
    acc = torch.zeros((54, 96, 4), dtype=torch.float32, device="cuda")
    m0 = cache.params()[0].copy()
    for f in range(8):
        st = cache.render(acc.data_ptr(), 96, 54, 1, seed=3, sample_offset=f, maxdepth=8, stats=True)
    torch.cuda.synchronize()
    img = acc.cpu().numpy()
    assert np.isfinite(img).all() and (img[..., 3] == 8).all()
    assert st["camera_samples"] == 96 * 54
    m1 = cache.params()[0]
    assert np.abs(m1 - m0).max() > 0          # the network was updated from the tracer's own samples
    assert gs.error_flags() == 0


def test_trained_cache_recovers_truncated_radiance(ctx):
    import torch
    from banshee_b200 import capi, scenes
    from banshee_b200 import convergence as CV
    from banshee_b200.metrics import relmse
    W = H = 64
    gs = capi.GpuScene(ctx, scenes.cornell(W, H))
    ref = CV.ground_truth(gs, W, H, 8192, 5, seed=99)

    def mean(acc):
        a = acc.double().cpu().numpy()
        return a[..., :3] / a[..., 3:4]

    frames = 256
    acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    gs.render(acc.data_ptr(), W, H, frames, seed=3, maxdepth=2, stats=False)
    torch.cuda.synchronize()
    e_trunc = relmse(mean(acc), ref)

    cache = capi.RadianceCache(gs, log2_table_size=16, base_resolution=8, max_resolution=256, train_paths=1024,
                               cache_depth=2, train_batch=4096, train_steps=2, learning_rate=1e-2)
    acc.zero_()
    for f in range(frames):
        cache.render(acc.data_ptr(), W, H, 1, seed=3, sample_offset=f, maxdepth=5)
    torch.cuda.synchronize()
    e_cache = relmse(mean(acc), ref)
    cache.close()

    acc.zero_()
    gs.render(acc.data_ptr(), W, H, frames, seed=3, maxdepth=5, stats=False)
    torch.cuda.synchronize()
    e_plain = relmse(mean(acc), ref)
    print("relMSE truncated %.3g cache %.3g plain %.3g" % (e_trunc, e_cache, e_plain))
    assert e_cache < 0.2 * e_trunc, (e_cache, e_trunc)
    assert e_cache < 3.0 * e_plain, (e_cache, e_plain)


def test_tcgen05_and_mma_sync_inference_agree(ctx):
    """The tcgen05 kernel (TMEM accumulators) and the mma.sync kernel compute the
    same bf16 network; only the fp32 summation order differs.  Ragged row counts
    exercise partial 128-row tiles; the largest gives every tile group of the
    tcgen05 kernel several tiles."""
    import torch
    from banshee_b200 import capi
    gs, c0 = _cache(ctx, log2t=12, mlp_kernel=0)
    c1 = capi.RadianceCache(gs, log2_table_size=12, base_resolution=4, max_resolution=64,
                            bbox=((0, 0, 0), (1, 1, 1)), mlp_kernel=1)
    m, g, _, _ = c0.params()
    c1.set_params(m, g)
    rng = np.random.default_rng(8)
    for n in (1, 127, 129, 5000, 65536 + 77, 300_005):
        fd = torch.from_numpy(_features(n, rng)).cuda()
        o0 = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        o1 = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        c0.query(fd.data_ptr(), o0.data_ptr(), n)
        c1.query(fd.data_ptr(), o1.data_ptr(), n)
        torch.cuda.synchronize()
        a, b = o0.cpu().numpy(), o1.cpu().numpy()
        assert np.isfinite(a).all() and (a[:, 3] == 0).all()
        scale = np.abs(b[:, :3]).max() + 1e-6
        assert np.abs(a[:, :3] - b[:, :3]).max() < 2e-2 * scale, (n, np.abs(a - b).max(), scale)
    assert gs.error_flags() == 0


@pytest.mark.parametrize("n", [3000 + 77, 65536 + 77])
def test_tcgen05_training_matches_mma_sync(ctx, n):
    """One training step's loss and gradients from the tcgen05 kernels (fused
    forward + backward, and the six weight-gradient GEMMs in one kernel) against
    the mma.sync kernels on the same rows: ragged counts (partial 128-row tiles
    and sample chunks), and enough rows that a CTA of the weight-gradient kernel
    accumulates several chunks.  Each weight matrix is compared on its own."""
    import torch
    from banshee_b200 import capi
    gs, c0 = _cache(ctx, log2t=10, mlp_kernel=0)
    c1 = capi.RadianceCache(gs, log2_table_size=10, base_resolution=4, max_resolution=64,
                            bbox=((0, 0, 0), (1, 1, 1)), mlp_kernel=1)
    rng = np.random.default_rng(12)
    m, g, _, _ = c0.params()
    g = (rng.random(g.shape).astype(np.float32) - 0.5) * 0.5
    c0.set_params(m, g)
    c1.set_params(m, g)
    feat = _features(n, rng)
    target = np.zeros((n, 4), np.float32)
    target[:, :3] = rng.random((n, 3))
    fd = torch.from_numpy(feat).cuda()
    td = torch.from_numpy(target).cuda()
    l0 = c0.train(fd.data_ptr(), td.data_ptr(), n, apply=False)
    l1 = c1.train(fd.data_ptr(), td.data_ptr(), n, apply=False)
    _, _, d0, dg0 = c0.params()
    _, _, d1, dg1 = c1.params()
    assert abs(l0 - l1) <= 1e-3 * abs(l1) + 1e-7, (l0, l1)
    # W0 [64 x 128], W1..W4 [64 x 64], W5 [16 x 64], then the hash grid
    bounds = [0, 8192, 12288, 16384, 20480, 24576, 25600]
    parts = [(d0[a:b], d1[a:b]) for a, b in zip(bounds[:-1], bounds[1:])] + [(dg0, dg1)]
    for k, (a, b) in enumerate(parts):
        a, b = a.astype(np.float64), b.astype(np.float64)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
        assert cos > 0.999 and np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30) < 2e-2, (k, cos)
    assert gs.error_flags() == 0


def test_new_cache_on_the_same_scene_gets_its_own_pass_graph(ctx):
    """A cached pass is captured into a CUDA graph that bakes in the cache's
    device buffers.  A cache created after another was destroyed (its host
    object and buffers possibly at the freed addresses, or not) must never
    replay the old cache's graph: its frames equal those of the same cache
    configuration on a fresh scene object."""
    import torch
    from banshee_b200 import capi, scenes
    sc = scenes.cornell(48, 48)
    cfg = dict(log2_table_size=12, base_resolution=4, max_resolution=64, train_paths=1024, cache_depth=2,
               train_batch=1024, train_steps=1, learning_rate=1e-2)

    def frames(gs, n=4):
        cache = capi.RadianceCache(gs, **cfg)
        acc = torch.zeros((48, 48, 4), dtype=torch.float32, device="cuda")
        for f in range(n):
            cache.render(acc.data_ptr(), 48, 48, 1, seed=5, sample_offset=f, maxdepth=5)
        torch.cuda.synchronize()
        cache.close()
        return acc.cpu().numpy()

    gs = capi.GpuScene(ctx, sc)
    frames(gs)                                                  # first cache: its graph is captured
    spacer = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")   # shifts later allocations
    again = frames(gs)                                          # second cache, same scene
    fresh = frames(capi.GpuScene(ctx, sc))
    del spacer
    assert np.isfinite(again).all() and (again[..., 3] == 4).all()
    from banshee_b200.metrics import mean_image, relmse
    # training uses float atomics, so the two runs agree to rounding, not bits
    assert relmse(mean_image(again), mean_image(fresh)) < 1e-2
    assert gs.error_flags() == 0


def test_two_caches_rendering_alternately_keep_their_own_networks(ctx):
    """Two caches of one configuration on one scene replay the same captured
    passes (graphs are keyed by the cache's configuration), each re-pointed at
    its own cache before every replay.  Rendering them alternately, each one's
    frames must match the same cache rendering alone on a scene object of its
    own; different network seeds make a mix-up visible."""
    import torch
    from banshee_b200 import capi, scenes
    from banshee_b200.metrics import mean_image, relmse
    sc = scenes.cornell(48, 48)
    cfg = dict(log2_table_size=12, base_resolution=4, max_resolution=64, train_paths=1024, cache_depth=2,
               train_batch=1024, train_steps=1, learning_rate=1e-2)

    def frames(caches, n=4):
        accs = [torch.zeros((48, 48, 4), dtype=torch.float32, device="cuda") for _ in caches]
        for f in range(n):
            for c, a in zip(caches, accs):
                c.render(a.data_ptr(), 48, 48, 1, seed=5, sample_offset=f, maxdepth=5)
        torch.cuda.synchronize()
        return [a.cpu().numpy() for a in accs]

    gs = capi.GpuScene(ctx, sc)
    a, b = capi.RadianceCache(gs, seed=1, **cfg), capi.RadianceCache(gs, seed=2, **cfg)
    both = frames([a, b])
    alone = [frames([capi.RadianceCache(capi.GpuScene(ctx, sc), seed=k, **cfg)])[0] for k in (1, 2)]
    for got, want in zip(both, alone):
        assert np.isfinite(got).all() and (got[..., 3] == 4).all()
        # training uses float atomics: the runs agree to rounding, not bits
        assert relmse(mean_image(got), mean_image(want)) < 1e-2
    # the two networks differ (different seeds), so each cache did read its own
    assert relmse(mean_image(both[0]), mean_image(both[1])) > relmse(mean_image(both[0]), mean_image(alone[0]))
    assert gs.error_flags() == 0
    a.close()
    b.close()
