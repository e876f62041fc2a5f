"""Render a few frames of a named workload, for profilers (ncu) and quick timing.

  python -m banshee_b200.profile_frames --workload c3 [--frames 1] [--width 8]
  python -m banshee_b200.profile_frames --workload c5 --frames 2
  python -m banshee_b200.profile_frames --workload c2 [--width 8]

c3: the 6.09M-triangle production scene at 1920x1080, plain GiTracer(8), --spp
    camera samples per pixel per frame (default 1: one pass of 2^21 paths;
    128-thread traversal blocks: no autotuning); k_trace launches per bounce
    are, in capture order, extension (closest hit) and shadow (any hit), plus
    MIS (closest hit) in scenes with area lights.
c5: the same scene through the radiance cache (2^19-entry hash grid levels,
    65,536 training paths per frame ending into the cache one bounce after the
    rendering paths, which end after 2 bounces; training one frame behind).
c2: the 1M-triangle soup, 16M incoherent closest-hit rays, one
    bg_intersect_closest call per frame.
Prints one JSON line with the CUDA-event time per frame.
"""
import argparse
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["c2", "c3", "c5"], default="c3")
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--width", type=int, default=0, help="node layout (4 or 8; 0 = scene default)")
    ap.add_argument("--spp", type=int, default=1, help="camera samples per pixel per frame (c3, c5)")
    args = ap.parse_args()
    import numpy as np
    import torch
    from . import capi, scenes
    ctx = capi.Context(0)
    t0 = time.perf_counter()
    if args.workload == "c2":
        sc = scenes.soup(1 << 20, seed=1)
    else:
        sc = scenes.production(1920, 1080)
    gs = capi.GpuScene(ctx, sc)
    if args.width:
        gs.set_node_width(args.width)
    build_s = time.perf_counter() - t0
    cache = None
    if args.workload == "c2":
        rays = scenes.soup_rays(1 << 24, "incoherent", seed=2)
        dr = torch.from_numpy(rays.view(np.uint8)).cuda()
        dh = torch.zeros((1 << 24) * 16, dtype=torch.uint8, device="cuda")

        def frame(f):
            gs.intersect_closest(dr.data_ptr(), dh.data_ptr(), 1 << 24)
    else:
        acc = torch.zeros((1080, 1920, 4), dtype=torch.float32, device="cuda")
        if args.workload == "c5":
            cache = capi.RadianceCache(gs, log2_table_size=19, base_resolution=16, max_resolution=2048,
                                       train_paths=65536, cache_depth=2, train_batch=65536, train_steps=1,
                                       learning_rate=1e-2, train_suffix=1)

            def frame(f):
                cache.render(acc.data_ptr(), 1920, 1080, args.spp, seed=1, sample_offset=f * args.spp, maxdepth=8)
        else:
            def frame(f):
                gs.render(acc.data_ptr(), 1920, 1080, args.spp, seed=1, sample_offset=f * args.spp, maxdepth=8,
                          stats=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for f in range(args.frames):
        frame(f)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"workload": args.workload, "frames": args.frames, "ms_per_frame": e0.elapsed_time(e1) / args.frames,
                      "node_width": gs.info()["node_width"], "build_s": build_s, "error_flags": gs.error_flags()}))
    if cache is not None:
        cache.close()


if __name__ == "__main__":
    main()
