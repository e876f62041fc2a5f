"""The optional watertight ray / triangle test (bg_build_opts.intersect = 1;
Woop, Benthin and Wald 2013).  It has no counterpart in the reference, whose
Moller-Trumbore test stays the default and the bit-exact one.

* parity: closest hits equal a float32 numpy restatement of the published
  algorithm (oracle/watertight.py) on the same rays, ids (exact-t ties
  classified), t and barycentrics bit for bit, on both node layouts;
* watertightness: rays from the centre of a closed sphere mesh aimed exactly
  at its vertices and at points on its shared edges never miss;
* agreement with Moller-Trumbore: the two tests pick the same triangle for all
  but edge cases, with t within 1e-5 relative.
"""
import numpy as np
import pytest

from banshee_b200 import abi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from banshee_b200 import capi
    return capi.Context(0)


def _verts(sc):
    m = sc.meshes[0]
    return np.ascontiguousarray(m.vertices[m.vidx.reshape(-1)].reshape(-1, 3, 3), dtype=np.float32)


@pytest.mark.parametrize("width", [4, 8])
def test_watertight_matches_restatement(ctx, width):
    from banshee_b200 import capi
    from oracle import watertight as WT
    sc = scenes.soup(10000, seed=17)
    gs = capi.GpuScene(ctx, sc, intersect=abi.BG_INTERSECT_WATERTIGHT)
    gs.set_node_width(width)
    rays = np.concatenate([scenes.soup_rays(2048, "incoherent", seed=18), scenes.soup_rays(1024, "coherent", seed=19)])
    got = gs.intersect_closest_host(rays)
    want = WT.intersect_closest(_verts(sc), rays)
    tie = (got["primid"] != want["primid"]) & (got["t"].view(np.uint32) == want["t"].view(np.uint32))
    assert ((got["primid"] == want["primid"]) | tie).all()
    assert (got["t"].view(np.uint32) == want["t"].view(np.uint32)).all()
    same = got["primid"] == want["primid"]
    assert (got["u"][same].view(np.uint32) == want["u"][same].view(np.uint32)).all()
    assert (got["v"][same].view(np.uint32) == want["v"][same].view(np.uint32)).all()
    occ = gs.intersect_any_host(scenes.soup_rays(2048, "incoherent", seed=20, any_hit=True))
    assert occ.sum() > 0
    assert gs.error_flags() == 0


def _sphere(nu=64, nv=32):
    """A closed UV sphere with shared vertices (poles shared by their fans)."""
    from banshee_b200.scene import Mesh, Scene, lambert
    v = [(0.0, 0.0, 1.0)]
    for j in range(1, nv):
        th = np.pi * j / nv
        for i in range(nu):
            ph = 2 * np.pi * i / nu
            v.append((np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)))
    v.append((0.0, 0.0, -1.0))
    ring = lambda j, i: 1 + (j - 1) * nu + (i % nu)
    f = []
    for i in range(nu):
        f.append((0, ring(1, i), ring(1, i + 1)))
        f.append((len(v) - 1, ring(nv - 1, i + 1), ring(nv - 1, i)))
    for j in range(1, nv - 1):
        for i in range(nu):
            a, b, c, d = ring(j, i), ring(j, i + 1), ring(j + 1, i), ring(j + 1, i + 1)
            f += [(a, c, b), (b, c, d)]
    v = np.array(v, np.float32) * np.float32(0.7) + np.float32(0.3)
    f = np.array(f, np.int32)
    m = Mesh(v, np.array([[0, 0, 1]], np.float32), f, np.zeros_like(f), np.zeros(len(f), np.int32))
    return Scene(meshes=[m], materials=[lambert((0.5, 0.5, 0.5))]), v, f


def test_rays_through_shared_vertices_and_edges_never_miss(ctx):
    from banshee_b200 import capi
    sc, v, f = _sphere()
    centre = np.float32(0.3)
    targets = [v]
    edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    for w in (0.5, 0.25, 0.125):
        targets.append((v[edges[:, 0]] * np.float32(w) + v[edges[:, 1]] * np.float32(1 - w)).astype(np.float32))
    tgt = np.concatenate(targets)
    rays = np.zeros(len(tgt), dtype=abi.RAY_DTYPE)
    rays["o"] = centre
    d = tgt - centre
    rays["d"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["tmax"] = np.float32(10.0)
    wt = capi.GpuScene(ctx, sc, intersect=abi.BG_INTERSECT_WATERTIGHT)
    for width in (4, 8):
        wt.set_node_width(width)
        hits = wt.intersect_closest_host(rays)
        assert (hits["primid"] >= 0).all(), int((hits["primid"] < 0).sum())
        assert wt.intersect_any_host(rays).all()
    mt = capi.GpuScene(ctx, sc).intersect_closest_host(rays)
    print("rays through vertices / edges that miss: watertight 0, Moller-Trumbore %d of %d"
          % (int((mt["primid"] < 0).sum()), len(rays)))
    assert wt.error_flags() == 0


def test_watertight_agrees_with_moller_trumbore_away_from_edges(ctx):
    from banshee_b200 import capi
    sc = scenes.soup(100_000, seed=21)
    rays = scenes.soup_rays(1 << 16, "incoherent", seed=22)
    mt = capi.GpuScene(ctx, sc).intersect_closest_host(rays)
    wt = capi.GpuScene(ctx, sc, intersect=abi.BG_INTERSECT_WATERTIGHT).intersect_closest_host(rays)
    same = (mt["primid"] == wt["primid"])
    assert same.mean() > 0.999, same.mean()
    h = same & (mt["primid"] >= 0)
    rel = np.abs(wt["t"][h] - mt["t"][h]) / np.abs(mt["t"][h])
    assert rel.max() < 1e-5, rel.max()
