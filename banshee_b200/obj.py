"""Wavefront OBJ / MTL reader -> Scene, for the reference's OBJ assets (such as
its Cornell box, 16 quads).

Follows what the reference's importer produces for an OBJ
(import/assimp_assetimporter.cpp:52-147): one Mesh per material group, faces
triangulated as fans, a Lambert material with the MTL's Kd, and for an
emissive material (non-zero Ke, or the material named "light") an Emissive
material with the importer's fixed emission 0.6 * (60, 55, 40) plus one
AreaLight per emissive triangle.  Missing normals become flat face normals,
missing texture coordinates (0, 0).
"""
import os

import numpy as np

from .scene import Mesh, Scene, area_light, emissive, lambert

REFERENCE_EMISSION = (0.6 * 60.0, 0.6 * 55.0, 0.6 * 40.0)


def _read_mtl(path):
    mats, cur = {}, None
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0].startswith("#"):
                continue
            if t[0] == "newmtl":
                cur = " ".join(t[1:])
                mats[cur] = {"Kd": (0.0, 0.0, 0.0), "Ke": (0.0, 0.0, 0.0)}
            elif cur is not None and t[0] in ("Kd", "Ke") and len(t) >= 4:
                mats[cur][t[0]] = tuple(float(x) for x in t[1:4])
    return mats


def load_obj(path, width=256, height=256, emission=REFERENCE_EMISSION):
    """Returns a Scene with meshes, materials and area lights (no camera)."""
    base = os.path.dirname(os.path.abspath(path))
    V, N, T = [], [], []
    groups = {}            # material name -> list of faces [(vi, ti, ni) * k]
    order = []
    mtl = {}
    cur = "default"
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0].startswith("#"):
                continue
            k = t[0]
            if k == "v":
                V.append([float(x) for x in t[1:4]])
            elif k == "vn":
                N.append([float(x) for x in t[1:4]])
            elif k == "vt":
                T.append([float(x) for x in t[1:3]])
            elif k == "mtllib":
                p = os.path.join(base, " ".join(t[1:]))
                if os.path.exists(p):
                    mtl.update(_read_mtl(p))
            elif k == "usemtl":
                cur = " ".join(t[1:])
            elif k == "f":
                face = []
                for item in t[1:]:
                    parts = item.split("/")
                    ix = [int(parts[j]) if j < len(parts) and parts[j] else 0 for j in range(3)]
                    # negative indices count back from the current end of the list
                    fix = [i - 1 if i > 0 else (len(lst) + i if i < 0 else -1)
                           for i, lst in zip(ix, (V, T, N))]
                    face.append(tuple(fix))
                if len(face) >= 3:
                    if cur not in groups:
                        groups[cur] = []
                        order.append(cur)
                    groups[cur].append(face)
    V = np.asarray(V, np.float32).reshape(-1, 3)
    N = np.asarray(N, np.float32).reshape(-1, 3)
    T = np.asarray(T, np.float32).reshape(-1, 2)
    sc = Scene(name=os.path.basename(path), width=width, height=height)
    for name in order:
        tris = []
        for face in groups[name]:
            for j in range(1, len(face) - 1):                 # fan triangulation
                tris.append((face[0], face[j], face[j + 1]))
        vi = np.array([[c[0] for c in tri] for tri in tris], np.int32)
        ti = np.array([[c[1] for c in tri] for tri in tris], np.int32)
        ni = np.array([[c[2] for c in tri] for tri in tris], np.int32)
        nf = vi.shape[0]
        if (ni < 0).any() or N.shape[0] == 0:
            p = V[vi]
            fn = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]).astype(np.float64)
            ln = np.linalg.norm(fn, axis=1, keepdims=True)
            fn = np.where(ln > 0, fn / np.maximum(ln, 1e-30), np.array([0.0, 0.0, 1.0])).astype(np.float32)
            normals, nidx = fn, np.repeat(np.arange(nf, dtype=np.int32)[:, None], 3, axis=1)
        else:
            normals, nidx = N, ni
        if (ti < 0).any() or T.shape[0] == 0:
            uvs, uidx = np.zeros((1, 2), np.float32), np.zeros((nf, 3), np.int32)
        else:
            uvs, uidx = T, ti
        m = mtl.get(name, {"Kd": (0.5, 0.5, 0.5), "Ke": (0.0, 0.0, 0.0)})
        is_light = any(x > 0.0 for x in m["Ke"]) or name == "light"
        midx = len(sc.materials)
        sc.materials.append(emissive(emission if emission is not None else m["Ke"]) if is_light
                            else lambert(m["Kd"]))
        sc.meshes.append(Mesh(V, normals, vi, nidx, np.full(nf, midx, np.int32), uvs, uidx))
        if is_light:
            sc.lights.extend(area_light(len(sc.meshes) - 1, f) for f in range(nf))
    return sc
