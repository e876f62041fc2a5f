"""Host-side scene description mirroring Banshee's World.

``Mesh`` mirrors the reference ``Mesh`` constructor (FireRays/Banshee/
primitive/mesh.h:69-76: separately indexed vertices, normals and uvs, one
material index per face) plus ``ShapeBundle::SetTransform``; ``Scene`` mirrors
``World``'s public fields (world/world.h:75-87: shapebundles_, materials_,
lights_, camera_, bgcolor_).  ``Scene.descs()`` packs everything into the
``bg_*_desc`` structs of include/banshee_gpu.h, which both the GPU library and
the CPU checker consume, so both see bit-identical inputs.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import ctypes as C
import numpy as np

from . import abi


@dataclass
class Mesh:
    vertices: np.ndarray            # (nv, 3) float32, object space
    normals: np.ndarray             # (nn, 3) float32
    vidx: np.ndarray                # (nf, 3) int32
    nidx: np.ndarray                # (nf, 3) int32
    materials: np.ndarray           # (nf,) int32
    uvs: Optional[np.ndarray] = None    # (nu, 2) float32
    uidx: Optional[np.ndarray] = None   # (nf, 3) int32
    m: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    minv: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float32).reshape(-1, 3)
        self.normals = np.ascontiguousarray(self.normals, dtype=np.float32).reshape(-1, 3)
        self.vidx = np.ascontiguousarray(self.vidx, dtype=np.int32).reshape(-1, 3)
        self.nidx = np.ascontiguousarray(self.nidx, dtype=np.int32).reshape(-1, 3)
        self.materials = np.ascontiguousarray(self.materials, dtype=np.int32).reshape(-1)
        if self.uvs is not None:
            self.uvs = np.ascontiguousarray(self.uvs, dtype=np.float32).reshape(-1, 2)
            self.uidx = np.ascontiguousarray(self.uidx, dtype=np.int32).reshape(-1, 3)
        self.m = np.ascontiguousarray(self.m, dtype=np.float32).reshape(4, 4)
        self.minv = np.ascontiguousarray(self.minv, dtype=np.float32).reshape(4, 4)

    @property
    def nfaces(self):
        return int(self.vidx.shape[0])

    def set_transform(self, m, minv=None):
        """ShapeBundle::SetTransform(m, minv); minv defaults to inverse(m) in float64."""
        m64 = np.asarray(m, dtype=np.float64).reshape(4, 4)
        self.m = m64.astype(np.float32)
        self.minv = (np.linalg.inv(m64) if minv is None else np.asarray(minv, dtype=np.float64)).astype(np.float32)

    def world_vertices(self):
        v = self.vertices.astype(np.float64)
        return (v @ self.m[:3, :3].astype(np.float64).T + self.m[:3, 3].astype(np.float64)).astype(np.float32)

    def desc(self):
        d = abi.MeshDesc()
        d.vertices = abi.fptr(self.vertices); d.nvertices = self.vertices.shape[0]; d.vstride = 0
        d.normals = abi.fptr(self.normals); d.nnormals = self.normals.shape[0]; d.nstride = 0
        if self.uvs is not None:
            d.uvs = abi.fptr(self.uvs); d.nuvs = self.uvs.shape[0]; d.ustride = 0
            d.uidx = abi.iptr(self.uidx); d.uistride = 0
        else:
            d.uvs = None; d.nuvs = 0; d.ustride = 0; d.uidx = None; d.uistride = 0
        d.vidx = abi.iptr(self.vidx); d.vistride = 0
        d.nidx = abi.iptr(self.nidx); d.nistride = 0
        d.materials = abi.iptr(self.materials); d.mstride = 4
        d.nfaces = self.nfaces
        d.m[:] = self.m.reshape(-1).tolist()
        d.minv[:] = self.minv.reshape(-1).tolist()
        return d


def lambert(kd):
    return dict(type=abi.BG_MAT_LAMBERT, kd=tuple(kd))


def ggx(roughness, eta=None, f0=None, ks=(1.0, 1.0, 1.0)):
    """Microfacet(eta, ks, FresnelDielectric, GgxDistribution(roughness)).

    A normal-incidence reflectance f0 is mapped to the dielectric index
    eta = (1 + sqrt(f0)) / (1 - sqrt(f0))."""
    if eta is None:
        s = float(np.sqrt(f0))
        eta = (1.0 + s) / (1.0 - s)
    return dict(type=abi.BG_MAT_MICROFACET_GGX, roughness=float(roughness), eta=float(eta), ks=tuple(ks))


def emissive(e):
    return dict(type=abi.BG_MAT_EMISSIVE, e=tuple(e))


def area_light(mesh, face):
    return dict(type=abi.BG_LIGHT_AREA, mesh=int(mesh), face=int(face))


def directional_light(d, e):
    return dict(type=abi.BG_LIGHT_DIRECTIONAL, d=tuple(d), e=tuple(e))


def environment_light(e, scale=1.0, gamma=1.0):
    return dict(type=abi.BG_LIGHT_ENVIRONMENT, e=tuple(e), scale=float(scale), gamma=float(gamma))


def camera(eye, at, up=(0.0, 1.0, 0.0), znear=0.01, zfar=10000.0, fovy_deg=40.0, aspect=1.0):
    return dict(eye=tuple(eye), at=tuple(at), up=tuple(up), znear=float(znear), zfar=float(zfar),
                fovy=float(np.float32(np.deg2rad(fovy_deg))), aspect=float(aspect))


@dataclass
class Scene:
    meshes: List[Mesh] = field(default_factory=list)
    materials: List[dict] = field(default_factory=list)
    lights: List[dict] = field(default_factory=list)
    bgcolor: tuple = (0.0, 0.0, 0.0)
    camera: Optional[dict] = None
    width: int = 256
    height: int = 256
    name: str = "scene"

    @property
    def ntriangles(self):
        return sum(m.nfaces for m in self.meshes)

    def descs(self):
        """(mesh array, n, material array, n, light array, n, bgcolor array); keep the result alive."""
        nm = len(self.meshes)
        marr = (abi.MeshDesc * max(nm, 1))()
        for i, m in enumerate(self.meshes):
            marr[i] = m.desc()
        mats = (abi.MaterialDesc * max(len(self.materials), 1))()
        for i, md in enumerate(self.materials):
            mats[i] = material_desc(md)
        lights = (abi.LightDesc * max(len(self.lights), 1))()
        for i, ld in enumerate(self.lights):
            lights[i] = light_desc(ld)
        bg = (C.c_float * 3)(*self.bgcolor)
        return marr, nm, mats, len(self.materials), lights, len(self.lights), bg

    def camera_desc(self):
        return camera_desc(self.camera)


def material_desc(md):
    d = abi.MaterialDesc()
    d.type = md["type"]
    d.kd[:] = list(md.get("kd", (0.0, 0.0, 0.0)))
    d.ks[:] = list(md.get("ks", (0.0, 0.0, 0.0)))
    d.eta = md.get("eta", 1.0)
    d.roughness = md.get("roughness", 0.0)
    d.e[:] = list(md.get("e", (0.0, 0.0, 0.0)))
    return d


def light_desc(ld):
    d = abi.LightDesc()
    d.type = ld["type"]
    d.mesh = ld.get("mesh", -1)
    d.face = ld.get("face", -1)
    d.d[:] = list(ld.get("d", (0.0, 0.0, 0.0)))
    d.e[:] = list(ld.get("e", (0.0, 0.0, 0.0)))
    d.scale = ld.get("scale", 1.0)
    d.gamma = ld.get("gamma", 1.0)
    return d


def camera_desc(c):
    d = abi.CameraDesc()
    d.eye[:] = list(c["eye"]); d.at[:] = list(c["at"]); d.up[:] = list(c["up"])
    d.znear = c["znear"]; d.zfar = c["zfar"]; d.fovy = c["fovy"]; d.aspect = c["aspect"]
    return d
