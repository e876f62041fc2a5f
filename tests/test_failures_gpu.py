"""Failure handling on the GPU, in forms that fault, trap or hang nothing.

* out of memory: the library's allocation cap (bg_alloc_limit) makes a scene
  commit and a render's path-state allocation fail as a failed cudaMalloc
  would; the call returns BG_ERR_OOM, keeps no partial state, and the same
  objects work once memory is available again;
* rays with NaN / Inf components, a zero direction or a NaN interval are
  misses, as in the reference's own Bvh (which the oracle restates); an
  infinite tmax is an ordinary interval.  A zero direction with an infinite
  tmax is degenerate: Moller-Trumbore's 0 * inf arithmetic lets a tested
  triangle report t = +inf, and which triangles get tested depends on the
  tree and on the slab test's rounding, so only t = +inf is required of it.
  Everything else equals the oracle's results, raises no device flag and
  leaves the other rays of the launch unaffected;
* a scene whose tree would need more traversal stack than a ray has is
  refused at commit (BG_ERR_UNSUPPORTED), so traversal never overflows;
* the tcgen05 kernels' bounded mbarrier waits: with a budget of one poll
  every wait gives up, the kernel raises BG_FLAG_TIMEOUT, drains its own MMA,
  frees its tensor memory and returns; the context stays usable and a cache
  with the default budget then gives the normal results.
The reference's error convention is an exception from the failing call
(light/arealight.cpp:18); across the C ABI that is a BG_ERR_* status.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BG_ERR_OOM, BG_ERR_STATE, BG_ERR_UNSUPPORTED = -3, -4, -7
BG_FLAG_TIMEOUT = 0x8


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


def test_commit_out_of_memory_leaves_no_state(ctx, oracle_built):
    from banshee_b200 import capi, scenes
    sc = scenes.soup(50_000, seed=31)
    gs = capi.GpuScene(ctx, sc, commit=False)
    capi.alloc_limit(1 << 20)                      # far below what the scene needs
    try:
        with pytest.raises(capi.BansheeError) as ei:
            gs.commit()
        assert ei.value.code == BG_ERR_OOM
    finally:
        capi.alloc_limit(None)
    # the failed commit left the scene uncommitted
    with pytest.raises(capi.BansheeError) as ei:
        gs.info()
    assert ei.value.code == BG_ERR_STATE
    # and the same scene commits once memory is there, with exact results
    gs.commit()
    rays = scenes.soup_rays(1 << 14, "incoherent", seed=32)
    got = gs.intersect_closest_host(rays)
    want = oracle_built.Oracle(sc).intersect_closest(rays)
    assert (got["primid"] == want["primid"]).all()
    assert gs.error_flags() == 0


def test_render_state_out_of_memory_then_identical_image(ctx):
    from banshee_b200 import capi, scenes
    sc = scenes.cornell(32, 32)
    gs = capi.GpuScene(ctx, sc)
    capi.alloc_limit(0)                            # the first render must allocate its path state
    try:
        with pytest.raises(capi.BansheeError) as ei:
            gs.render_host(32, 32, 2, seed=3, maxdepth=5)
        assert ei.value.code == BG_ERR_OOM
    finally:
        capi.alloc_limit(None)
    img = gs.render_host(32, 32, 2, seed=3, maxdepth=5)
    ref = capi.GpuScene(ctx, sc).render_host(32, 32, 2, seed=3, maxdepth=5)
    assert (img.view(np.uint32) == ref.view(np.uint32)).all()
    assert gs.error_flags() == 0


def _bad_rays(n=4096):
    from banshee_b200 import scenes
    rays = scenes.soup_rays(n, "incoherent", seed=9)
    nan, inf = np.float32(np.nan), np.float32(np.inf)
    rays["o"][0] = (nan, 0.5, 0.5)
    rays["d"][1] = (nan, 0.0, 1.0)
    rays["o"][2] = (inf, 0.5, 0.5)
    rays["d"][3] = (inf, 0.0, 0.0)
    rays["d"][4] = (0.0, 0.0, 0.0)
    rays["tmin"][5] = nan
    rays["tmax"][6] = nan
    rays["d"][7] = (-inf, inf, 0.0)
    rays["o"][8] = (-inf, -inf, -inf)
    rays["tmax"][9] = inf                       # an ordinary ray with an unbounded interval
    rays["d"][10] = (0.0, 0.0, 0.0)             # zero direction, unbounded: ties at t = +inf
    rays["tmax"][10] = inf
    return rays, 9                              # rays 0..8 must miss


@pytest.mark.parametrize("width", [4, 8])
def test_nan_inf_and_zero_direction_rays_miss(ctx, oracle_built, width):
    from banshee_b200 import capi, scenes
    sc = scenes.soup(200_000, seed=4)
    gs = capi.GpuScene(ctx, sc)
    gs.set_node_width(width)
    rays, nbad = _bad_rays()
    from tests.test_raycast_gpu import classify
    o = oracle_built.Oracle(sc)
    got = gs.intersect_closest_host(rays)
    want = o.intersect_closest(rays)
    assert (got["primid"][:nbad] == -1).all()
    assert got["t"][10] == np.inf                  # the degenerate zero-direction, unbounded ray
    keep = np.ones(rays.shape[0], bool)
    keep[10] = False
    ties, bad = classify(o, rays[keep], got[keep], want[keep])
    assert not bad, bad
    assert (got["t"][keep].view(np.uint32) == want["t"][keep].view(np.uint32)).all()
    occ = gs.intersect_any_host(rays)
    assert (occ[:nbad] == 0).all()
    assert (occ[keep] == o.intersect_any(rays)[keep]).all()
    assert (got["primid"][nbad:] >= 0).any()       # the ordinary rays of the launch still hit
    assert gs.error_flags() == 0


def _caterpillar(n=300, r=0.8):
    """Triangles k = 0..n-1 inside [r^k / 2, r^k]^3: each one nests the rest,
    so every split peels one triangle off and the tree is n levels deep."""
    from banshee_b200.scene import Mesh, Scene, lambert
    v, idx = [], []
    for k in range(n):
        s = r ** k
        v += [(0.5 * s, 0.5 * s, 0.5 * s), (s, 0.5 * s, 0.75 * s), (0.75 * s, s, s)]
        idx.append((3 * k, 3 * k + 1, 3 * k + 2))
    m = Mesh(np.array(v, np.float32), np.array([[0, 0, 1]], np.float32), np.array(idx, np.int32),
             np.zeros((n, 3), np.int32), np.zeros(n, np.int32))
    return Scene(meshes=[m], materials=[lambert((0.5, 0.5, 0.5))])


def test_tree_deeper_than_the_traversal_stack_is_refused_at_commit(ctx):
    from banshee_b200 import capi
    gs = capi.GpuScene(ctx, _caterpillar(), max_leaf=1, node_width=4, commit=False)
    with pytest.raises(capi.BansheeError) as ei:
        gs.commit()
    assert ei.value.code == BG_ERR_UNSUPPORTED and "stack" in str(ei.value)
    with pytest.raises(capi.BansheeError) as ei:
        gs.info()
    assert ei.value.code == BG_ERR_STATE


def test_tcgen05_bounded_wait_times_out_and_context_survives(ctx):
    import torch
    from banshee_b200 import capi, scenes
    from tests.test_cache_gpu import _features
    gs = capi.GpuScene(ctx, scenes.cornell(8, 8))
    kw = dict(log2_table_size=8, base_resolution=4, max_resolution=64, bbox=((0, 0, 0), (1, 1, 1)), mlp_kernel=0)
    n = 4096
    feat = torch.from_numpy(_features(n, np.random.default_rng(5))).cuda()
    out = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    quick = capi.RadianceCache(gs, wait_polls=1, **kw)
    gs.error_flags(clear=True)
    quick.query(feat.data_ptr(), out.data_ptr(), n)
    torch.cuda.synchronize()
    assert gs.error_flags(clear=True) & BG_FLAG_TIMEOUT
    # the context is still usable: the same parameters with the default budget
    normal = capi.RadianceCache(gs, **kw)
    normal.set_params(*quick.params()[:2])
    out.zero_()
    normal.query(feat.data_ptr(), out.data_ptr(), n)
    ref = torch.zeros_like(out)
    slow = capi.RadianceCache(gs, **dict(kw, mlp_kernel=1))       # mma.sync path: no mbarrier waits
    slow.set_params(*quick.params()[:2])
    slow.query(feat.data_ptr(), ref.data_ptr(), n)
    torch.cuda.synchronize()
    assert gs.error_flags() == 0
    o, r = out.cpu().numpy()[:, :3], ref.cpu().numpy()[:, :3]
    assert np.isfinite(o).all()
    err = np.abs(o - r).max() / (np.abs(r).max() + 1e-12)      # the forward tolerance of test_cache_gpu
    assert err < 2e-2, err
