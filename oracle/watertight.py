"""Watertight ray / triangle test restated in numpy float32 -- TEST INFRASTRUCTURE ONLY.

The library's optional watertight mode (bg_build_opts.intersect = 1) has no
counterpart in the reference, whose only test is Moller-Trumbore
(primitive/mesh.cpp:7-45).  This is the checker for that mode: the published
algorithm of Woop, Benthin and Wald, "Watertight Ray/Triangle Intersection",
JCGT 2(1), 2013, evaluated operation by operation in float32 (numpy rounds
every float32 operation and fuses none, as the library is compiled), with the
paper's double-precision recomputation of edge functions that come out 0.
Closest hit by brute force over all triangles, for small scenes only.
"""
import numpy as np

from banshee_b200 import abi

f32 = np.float32


def _shear(d):
    """kx, ky, kz and sx, sy, sz per ray (d: (n, 3) float32)."""
    ad = np.abs(d)
    kz = np.where((ad[:, 0] >= ad[:, 1]) & (ad[:, 0] >= ad[:, 2]), 0, np.where(ad[:, 1] >= ad[:, 2], 1, 2))
    kx = np.where(kz == 2, 0, kz + 1)
    ky = np.where(kx == 2, 0, kx + 1)
    n = np.arange(d.shape[0])
    dz = d[n, kz]
    swap = dz < 0
    kx, ky = np.where(swap, ky, kx), np.where(swap, kx, ky)
    sx = (d[n, kx] / dz).astype(f32)
    sy = (d[n, ky] / dz).astype(f32)
    sz = (f32(1.0) / dz).astype(f32)
    return kx, ky, kz, sx, sy, sz


def intersect_closest(verts, rays):
    """verts: (T, 3, 3) float32 triangle vertices in world space (identity
    bundles only); rays: bg_ray structured array.  Returns a bg_hit array."""
    o = np.ascontiguousarray(rays["o"], dtype=f32)
    d = np.ascontiguousarray(rays["d"], dtype=f32)
    tmin = rays["tmin"].astype(f32)
    n = rays.shape[0]
    kx, ky, kz, sx, sy, sz = _shear(d)
    hits = np.zeros(n, dtype=abi.HIT_DTYPE)
    hits["t"] = rays["tmax"]
    hits["primid"] = -1
    idx = np.arange(n)
    for tri in range(verts.shape[0]):
        P = verts[tri]                                       # (3, 3)
        rel = [(P[k][None, :] - o).astype(f32) for k in range(3)]      # A, B, C: (n, 3)
        z = [r[idx, kz] for r in rel]
        xy = [((r[idx, kx] - (sx * zz).astype(f32)).astype(f32), (r[idx, ky] - (sy * zz).astype(f32)).astype(f32))
              for r, zz in zip(rel, z)]
        (ax, ay), (bx, by), (cx, cy) = xy
        U = ((cx * by).astype(f32) - (cy * bx).astype(f32)).astype(f32)
        V = ((ax * cy).astype(f32) - (ay * cx).astype(f32)).astype(f32)
        W = ((bx * ay).astype(f32) - (by * ax).astype(f32)).astype(f32)
        zero = (U == 0) | (V == 0) | (W == 0)
        if zero.any():
            dd = lambda a: a.astype(np.float64)
            U = np.where(zero, (dd(cx) * dd(by) - dd(cy) * dd(bx)).astype(f32), U)
            V = np.where(zero, (dd(ax) * dd(cy) - dd(ay) * dd(cx)).astype(f32), V)
            W = np.where(zero, (dd(bx) * dd(ay) - dd(by) * dd(ax)).astype(f32), W)
        out = ((U < 0) | (V < 0) | (W < 0)) & ((U > 0) | (V > 0) | (W > 0))
        det = ((U + V).astype(f32) + W).astype(f32)
        with np.errstate(divide="ignore", invalid="ignore"):
            az, bz, cz = ((sz * zz).astype(f32) for zz in z)
            T = (((U * az).astype(f32) + (V * bz).astype(f32)).astype(f32) + (W * cz).astype(f32)).astype(f32)
            rcp = (f32(1.0) / det).astype(f32)
            t = (T * rcp).astype(f32)
            a = (V * rcp).astype(f32)
            b = (W * rcp).astype(f32)
        ok = ~out & (det != 0) & (t > tmin) & (t <= hits["t"])
        hits["t"] = np.where(ok, t, hits["t"])
        hits["primid"] = np.where(ok, tri, hits["primid"])
        hits["u"] = np.where(ok, a, hits["u"])
        hits["v"] = np.where(ok, b, hits["v"])
    return hits
