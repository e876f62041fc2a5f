"""Regenerate the golden fixtures in this directory from Banshee's own code.

Runs the reference sources compiled unmodified (oracle/_ref/libbanshee_ref.so,
built by ``make -C oracle ref`` where the reference tree is present) on small
seeded scenes and stores inputs + outputs as .npz:

  raycast_soup.npz      -- 20k-triangle soup; incoherent / coherent closest-hit
                           rays (primid, t, u, v) and incoherent any-hit rays
  raycast_cornell.npz   -- Cornell box (transformed bundles) camera rays
  render_cornell.npz    -- Cornell 32x32, 8 spp, GiTracer(5) and DiTracer images
  render_production.npz -- small production scene (GGX, sun, environment),
                           48x27, 4 spp, GiTracer(8)
  render_samplers.npz   -- Cornell 32x32: GiTracer(5) with the Sobol and the
                           CMJ (grid 4, from sample 3) image samplers, and
                           AoTracer(0.25) with the random and Sobol samplers

Usage:  python tests/golden/make_golden.py [--only samplers]
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from banshee_b200 import abi, scenes  # noqa: E402
from oracle.oracle import Reference  # noqa: E402


def scene_hash(sc):
    h = hashlib.sha256()
    for m in sc.meshes:
        for a in (m.vertices, m.normals, m.vidx, m.nidx, m.materials, m.m, m.minv):
            h.update(np.ascontiguousarray(a).tobytes())
        if m.uvs is not None:
            h.update(m.uvs.tobytes()); h.update(m.uidx.tobytes())
    return h.hexdigest()


SOUP = dict(ntris=20000, seed=3)
CORNELL = dict(width=32, height=32)
PROD = dict(width=48, height=27, nterrain=48, nspheres=12, sphere_seg=12, seed=3)


def samplers():
    cb = scenes.cornell(**CORNELL)
    refr = Reference(cb)
    out = {"scene_sha256": np.array(scene_hash(cb))}
    out["gi_sobol"] = refr.render(spp=8, seed=4, tracer=abi.BG_TRACER_GI, maxdepth=5, nthreads=1,
                                  sampler=abi.BG_SAMPLER_SOBOL)
    out["gi_cmj4"] = refr.render(spp=8, seed=4, tracer=abi.BG_TRACER_GI, maxdepth=5, nthreads=1,
                                 sampler=abi.BG_SAMPLER_CMJ, grid=4, sample_offset=3)
    out["ao"] = refr.render(spp=8, seed=4, tracer=abi.BG_TRACER_AO, maxdepth=1, nthreads=1, ao_radius=0.25)
    out["ao_sobol"] = refr.render(spp=8, seed=4, tracer=abi.BG_TRACER_AO, maxdepth=1, nthreads=1, ao_radius=0.25,
                                  sampler=abi.BG_SAMPLER_SOBOL)
    np.savez_compressed(os.path.join(HERE, "render_samplers.npz"), spp=8, seed=4, maxdepth=5, ao_radius=0.25,
                        cmj_grid=4, cmj_offset=3, **out)


def main():
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "samplers":
        samplers()
        print("golden fixtures written to", HERE)
        return
    samplers()
    sc = scenes.soup(**SOUP)
    ref = Reference(sc, raycast=True)
    out = {"scene_sha256": np.array(scene_hash(sc))}
    for kind, seed in (("incoherent", 5), ("coherent", 6)):
        rays = scenes.soup_rays(64 * 64, kind, seed=seed)
        hits = ref.intersect_closest(rays, nthreads=1)
        out[kind + "_rays"] = rays
        out[kind + "_hits"] = hits
    arays = scenes.soup_rays(64 * 64, "incoherent", seed=7, any_hit=True)
    out["any_rays"] = arays
    out["any_occluded"] = ref.intersect_any(arays, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "raycast_soup.npz"), **out)

    cb = scenes.cornell(**CORNELL)
    refc = Reference(cb, raycast=True)
    rng = np.random.default_rng(11)
    from oracle.oracle import Oracle
    cam_rays = Oracle(cb).camera_rays(rng.random((4096, 2)))
    np.savez_compressed(os.path.join(HERE, "raycast_cornell.npz"), scene_sha256=np.array(scene_hash(cb)),
                        rays=cam_rays, hits=refc.intersect_closest(cam_rays, nthreads=1))

    refr = Reference(cb)
    gi = refr.render(spp=8, seed=1, tracer=abi.BG_TRACER_GI, maxdepth=5, nthreads=1)
    di = refr.render(spp=8, seed=1, tracer=abi.BG_TRACER_DI, maxdepth=1, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "render_cornell.npz"), scene_sha256=np.array(scene_hash(cb)),
                        gi=gi, di=di, spp=8, seed=1, maxdepth=5)

    sp = scenes.production(**PROD)
    refp = Reference(sp)
    gi = refp.render(spp=4, seed=2, tracer=abi.BG_TRACER_GI, maxdepth=8, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "render_production.npz"), scene_sha256=np.array(scene_hash(sp)),
                        gi=gi, spp=4, seed=2, maxdepth=8)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
