"""Seeded procedural scenes for the five benchmark configurations.

All generators are deterministic in ``seed`` (numpy PCG64) and return
``scene.Scene`` objects that feed both the GPU library and the CPU checker.

* ``cornell``     -- C1: Cornell box, 5 wall quads + tall/short boxes = 34
  triangles, plus a 0.25 x 0.25 ceiling quad light (2 emissive triangles, so
  36 triangles in the BVH; the light is counted separately from the 34).
  The boxes carry bundle transforms (rotation about y + translation), so the
  per-bundle ray transform of Mesh::IntersectShape (primitive/mesh.cpp:224-228)
  is exercised.
* ``soup``        -- C2: triangle soup in the unit cube (centroids uniform,
  vertex offsets a random unit direction times U[0.001, 0.01]).
* ``soup_rays``   -- C2 ray sets: coherent pinhole rays aimed at the cube and
  incoherent rays (origins in the cube, directions uniform on the sphere).
* ``production``  -- C3: fractal (fBm) terrain heightfield plus UV spheres as
  separate transformed mesh bundles; GGX / Lambert materials; a sun
  (DirectionalLight) and a constant EnvironmentLight.
* ``batch``       -- C4: many production-style scenes of uneven size.
"""
import math

import numpy as np

from . import abi
from .scene import (Mesh, Scene, area_light, camera, directional_light, emissive,
                    environment_light, ggx, lambert)

FLT_MAX = float(np.finfo(np.float32).max)


def _rot_y(deg):
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]], dtype=np.float64)


def _translate(t):
    m = np.eye(4)
    m[:3, 3] = t
    return m


def _scale(s):
    m = np.eye(4)
    m[0, 0] = m[1, 1] = m[2, 2] = s
    return m


def _quad(p0, p1, p2, p3, n):
    """Two triangles (p0,p1,p2), (p0,p2,p3) with a flat normal n."""
    v = np.array([p0, p1, p2, p3], dtype=np.float32)
    return v, np.array([n], dtype=np.float32), np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)


def _merge(parts, mats):
    verts, norms, vidx, nidx, mids = [], [], [], [], []
    vo = no = 0
    for (v, n, f), m in zip(parts, mats):
        verts.append(v); norms.append(n)
        vidx.append(f + vo)
        nidx.append(np.full_like(f, no))
        mids.append(np.full(f.shape[0], m, dtype=np.int32))
        vo += v.shape[0]; no += n.shape[0]
    return Mesh(np.concatenate(verts), np.concatenate(norms), np.concatenate(vidx),
                np.concatenate(nidx), np.concatenate(mids))


def _box_mesh(sx, sy, sz, mat):
    """Axis-aligned box [-sx/2, sx/2] x [0, sy] x [-sz/2, sz/2], outward normals, 12 triangles."""
    x0, x1, z0, z1 = -sx / 2, sx / 2, -sz / 2, sz / 2
    y0, y1 = 0.0, sy
    parts = [
        _quad((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0), (0, 1, 0)),    # top
        _quad((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1), (0, -1, 0)),   # bottom
        _quad((x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1), (0, 0, 1)),    # front
        _quad((x1, y0, z0), (x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (0, 0, -1)),   # back
        _quad((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0), (-1, 0, 0)),   # left
        _quad((x1, y0, z1), (x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (1, 0, 0)),    # right
    ]
    return _merge(parts, [mat] * 6)


def cornell(width=256, height=256):
    """C1 Cornell box in [0,1]^3, open towards +z where the camera sits."""
    white, red, green, light = 0, 1, 2, 3
    walls = _merge([
        _quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0)),      # floor
        _quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0), (0, -1, 0)),     # ceiling
        _quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0), (0, 0, 1)),      # back
        _quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), (1, 0, 0)),      # left (red)
        _quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), (-1, 0, 0)),     # right (green)
    ], [white, white, white, red, green])
    tall = _box_mesh(0.33, 0.6, 0.33, white)
    tall.set_transform(_translate((0.33, 0.0, 0.37)) @ _rot_y(15.0))
    short = _box_mesh(0.33, 0.33, 0.33, white)
    short.set_transform(_translate((0.67, 0.0, 0.65)) @ _rot_y(-18.0))
    h = 0.999
    lq = _merge([_quad((0.375, h, 0.375), (0.375, h, 0.625), (0.625, h, 0.625), (0.625, h, 0.375),
                       (0, -1, 0))], [light])
    sc = Scene(name="cornell", width=width, height=height)
    sc.meshes = [walls, tall, short, lq]
    sc.materials = [lambert((0.73, 0.73, 0.73)), lambert((0.65, 0.05, 0.05)),
                    lambert((0.12, 0.45, 0.15)), emissive((15.0, 15.0, 15.0))]
    sc.lights = [area_light(3, 0), area_light(3, 1)]
    sc.camera = camera((0.5, 0.5, 2.4), (0.5, 0.5, 0.0), (0, 1, 0), 0.01, 100.0, 40.0, width / height)
    return sc


def soup(ntris=1 << 20, seed=1):
    """C2 triangle soup: one mesh, identity transform, one flat normal per face."""
    rng = np.random.default_rng(seed)
    c = rng.random((ntris, 3))
    d = rng.normal(size=(ntris, 3, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    r = rng.uniform(0.001, 0.01, size=(ntris, 3, 1))
    v = (c[:, None, :] + d * r).astype(np.float32)
    n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]).astype(np.float64)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(ln > 0, n / np.maximum(ln, 1e-30), np.array([0.0, 0.0, 1.0]))
    idx = np.arange(3 * ntris, dtype=np.int32).reshape(ntris, 3)
    nidx = np.repeat(np.arange(ntris, dtype=np.int32)[:, None], 3, axis=1)
    mesh = Mesh(v.reshape(-1, 3), n.astype(np.float32), idx, nidx, np.zeros(ntris, np.int32))
    sc = Scene(name="soup%d" % ntris)
    sc.meshes = [mesh]
    sc.materials = [lambert((0.5, 0.5, 0.5))]
    return sc


def soup_rays(nrays=1 << 24, kind="incoherent", seed=2, any_hit=False, tmax_range=(0.0, 1.0)):
    """C2 rays.  coherent: a pinhole grid of sqrt(n) x sqrt(n) rays from (0.5,0.5,2.5)
    at the cube centre; incoherent: origins U[0,1]^3, directions uniform on S^2.
    tmin = 0; tmax = FLT_MAX for closest-hit sets, U[tmax_range] (default U[0,1],
    the config's shadow interval) for any-hit sets.  Coherent rays start 1.5
    units in front of the cube, so coherent any-hit rays with tmax in [0,1]
    end before reaching it; tmax_range=(1.5, 2.5) makes them end inside it."""
    rng = np.random.default_rng(seed)
    rays = np.zeros(nrays, dtype=abi.RAY_DTYPE)
    if kind == "coherent":
        side = int(round(math.sqrt(nrays)))
        assert side * side == nrays
        eye = np.array([0.5, 0.5, 2.5])
        half = math.tan(math.radians(45.0) / 2)
        j, i = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
        x = ((i + 0.5) / side * 2 - 1) * half
        y = (1 - (j + 0.5) / side * 2) * half
        d = np.stack([x, y, -np.ones_like(x)], axis=-1).reshape(-1, 3)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rays["o"] = eye.astype(np.float32)
        rays["d"] = d.astype(np.float32)
    else:
        rays["o"] = rng.random((nrays, 3)).astype(np.float32)
        d = rng.normal(size=(nrays, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rays["d"] = d.astype(np.float32)
    rays["tmin"] = 0.0
    if any_hit:
        lo, hi = tmax_range
        rays["tmax"] = (lo + (hi - lo) * rng.random(nrays)).astype(np.float32)
    else:
        rays["tmax"] = FLT_MAX
    return rays


# ------------------------------------------------------------------ terrain
def _fbm(n, octaves, rng):
    """Value-noise fBm on an n x n grid in [0,1)^2, amplitude ~1."""
    u = np.linspace(0.0, 1.0, n, endpoint=False)
    h = np.zeros((n, n))
    amp, freq, total = 1.0, 4, 0.0
    for _ in range(octaves):
        lat = rng.random((freq + 1, freq + 1)) * 2 - 1
        x = u * freq
        i0 = np.floor(x).astype(np.int64)
        f = x - i0
        f = f * f * (3 - 2 * f)
        a = lat[np.ix_(i0, i0)] * (1 - f)[:, None] + lat[np.ix_(i0 + 1, i0)] * f[:, None]
        b = lat[np.ix_(i0, i0 + 1)] * (1 - f)[:, None] + lat[np.ix_(i0 + 1, i0 + 1)] * f[:, None]
        h += amp * (a * (1 - f)[None, :] + b * f[None, :])
        total += amp
        amp *= 0.5
        freq *= 2
    return h / total


def terrain_mesh(n, extent, height, rng, material):
    """n x n vertex heightfield over [-extent, extent]^2 -> 2 (n-1)^2 triangles,
    smooth finite-difference vertex normals and grid uvs."""
    h = _fbm(n, 8, rng) * height
    g = np.linspace(-extent, extent, n)
    X, Z = np.meshgrid(g, g, indexing="ij")
    verts = np.stack([X, h, Z], axis=-1).reshape(-1, 3).astype(np.float32)
    dx = np.gradient(h, g, axis=0)
    dz = np.gradient(h, g, axis=1)
    nrm = np.stack([-dx, np.ones_like(h), -dz], axis=-1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    uv = np.stack(np.meshgrid(np.arange(n) / (n - 1), np.arange(n) / (n - 1), indexing="ij"), -1)
    i = np.arange(n - 1)
    I, J = np.meshgrid(i, i, indexing="ij")
    a = (I * n + J).reshape(-1)
    b, c, d = a + n, a + n + 1, a + 1
    faces = np.empty((2 * a.size, 3), dtype=np.int32)
    faces[0::2] = np.stack([a, b, c], 1)
    faces[1::2] = np.stack([a, c, d], 1)
    mesh = Mesh(verts, nrm.reshape(-1, 3).astype(np.float32), faces, faces,
                np.full(faces.shape[0], material, np.int32),
                uv.reshape(-1, 2).astype(np.float32), faces)
    return mesh, h, g


def uv_sphere(nseg=100, nbands=101):
    """Unit UV sphere: 2 * nseg cap triangles + 2 * nseg * (nbands - 2) band
    triangles (100 x 101 -> 20,000), vertex normals = positions, (phi, theta) uvs."""
    th = np.pi * np.arange(1, nbands) / nbands            # nbands-1 rings
    ph = 2 * np.pi * np.arange(nseg + 1) / nseg           # seam duplicated
    T, P = np.meshgrid(th, ph, indexing="ij")
    ring = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    ruv = np.stack([P / (2 * np.pi), T / np.pi], -1).reshape(-1, 2)
    nr = nbands - 1
    top = np.array([[0.0, 1.0, 0.0]] * nseg)
    bot = np.array([[0.0, -1.0, 0.0]] * nseg)
    tuv = np.stack([(np.arange(nseg) + 0.5) / nseg, np.zeros(nseg)], -1)
    buv = np.stack([(np.arange(nseg) + 0.5) / nseg, np.ones(nseg)], -1)
    verts = np.concatenate([ring, top, bot]).astype(np.float32)
    uvs = np.concatenate([ruv, tuv, buv]).astype(np.float32)
    W = nseg + 1
    tb, bb = nr * W, nr * W + nseg
    faces = []
    s = np.arange(nseg)
    faces.append(np.stack([tb + s, s + 1, s], 1))                       # top cap
    for r in range(nr - 1):
        a = r * W + s
        faces.append(np.stack([a, a + 1, a + W + 1], 1))
        faces.append(np.stack([a, a + W + 1, a + W], 1))
    a = (nr - 1) * W + s
    faces.append(np.stack([bb + s, a, a + 1], 1))                       # bottom cap
    faces = np.concatenate(faces).astype(np.int32)
    return verts, uvs, faces


def production(width=1920, height=1080, nterrain=1024, nspheres=200, sphere_seg=100, seed=1):
    """C3: terrain (nterrain^2 grid) + nspheres UV spheres (separate bundles with
    translate+scale transforms, radius U[0.5,3]); sphere materials 70% GGX
    (roughness U[0.05,0.8], F0 U[0.02,0.9]) / 30% Lambert; terrain Lambert; a sun and
    a constant environment."""
    rng = np.random.default_rng(seed)
    extent = 64.0
    sc = Scene(name="production", width=width, height=height)
    sc.materials = [lambert((0.5, 0.45, 0.4))]
    terrain, h, g = terrain_mesh(nterrain, extent, 6.0, rng, 0)
    sc.meshes = [terrain]
    sv, suv, sf = uv_sphere(sphere_seg, sphere_seg + 1)
    for k in range(nspheres):
        if rng.random() < 0.7:
            sc.materials.append(ggx(rng.uniform(0.05, 0.8), f0=rng.uniform(0.02, 0.9)))
        else:
            sc.materials.append(lambert(tuple(rng.uniform(0.2, 0.9, 3))))
        mid = len(sc.materials) - 1
        r = rng.uniform(0.5, 3.0)
        x, z = rng.uniform(-0.8 * extent, 0.8 * extent, 2)
        ix = int(np.clip(np.searchsorted(g, x), 0, len(g) - 1))
        iz = int(np.clip(np.searchsorted(g, z), 0, len(g) - 1))
        y = float(h[ix, iz]) + 0.8 * r
        m = Mesh(sv, sv, sf, sf, np.full(sf.shape[0], mid, np.int32), suv, sf)
        m.set_transform(_translate((x, y, z)) @ _scale(r))
        sc.meshes.append(m)
    sc.lights = [directional_light((-0.35, -1.0, -0.25), (2.8, 2.6, 2.3)),
                 environment_light((0.25, 0.3, 0.4), 1.0, 1.0)]
    sc.camera = camera((0.0, 28.0, 75.0), (0.0, 0.0, 0.0), (0, 1, 0), 0.01, 10000.0, 60.0, width / height)
    return sc


def batch(nscenes=64, seed=7, tri_lo=1e4, tri_hi=5e5):
    """C4: production-style scenes with log-uniform triangle counts, resolutions
    from {256^2, 512^2, 1024x768} and spp U{16..128}.  Returns [(scene, spp)]."""
    rng = np.random.default_rng(seed)
    res = [(256, 256), (512, 512), (1024, 768)]
    out = []
    for k in range(nscenes):
        T = float(np.exp(rng.uniform(np.log(tri_lo), np.log(tri_hi))))
        w, hgt = res[int(rng.integers(0, 3))]
        spp = int(rng.integers(16, 129))
        nsph = int(rng.integers(4, 24))
        seg = max(8, int(math.sqrt(0.4 * T / nsph / 2)))
        tris_s = nsph * 2 * seg * seg
        n = max(8, int(math.sqrt(max(T - tris_s, 2e3) / 2)) + 1)
        sc = production(w, hgt, nterrain=n, nspheres=nsph, sphere_seg=seg, seed=int(rng.integers(1 << 30)))
        sc.name = "batch%02d" % k
        out.append((sc, spp))
    return out
