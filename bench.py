#!/usr/bin/env python
"""Benchmark: plain wavefront GI tracer at 1080p on the production scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one pass of the hot path over one batch: every pixel of a
1920x1080 frame gets one camera sample traced by GiTracer(8) (Russian roulette
after bounce 3) on the seeded 6.09M-triangle production scene (fBm terrain +
200 transformed UV spheres, GGX / Lambert, sun + constant environment).
Prints ONE JSON line (rank 0).  N > 1 runs under torchrun, one rank per GPU:
each rank traces its own samples of the frame (weak scaling) into a per-step
RGBW buffer; one NCCL all-reduce per step sums the ranks' step buffers, and the
sum is added once into the running image.

--impl reference times Banshee's own CPU tracer (the reference sources compiled
unmodified in oracle/_ref) on the box's host cores on a bounded sample of the
same workload: every step renders a band of rows of the same frame at 1 spp
with all host threads.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WIDTH, HEIGHT, MAXDEPTH, SEED = 1920, 1080, 8, 1
SPP = 8   # camera samples per pixel per step: the 256-spp image in 32 steps
METRIC = "Msamples/s at 1080p"
WORKLOAD = ("C3 plain wavefront GI tracer: seeded fBm terrain (1024^2 grid) + 200 UV spheres "
            "(20k triangles each, own transforms) = 6.09M triangles, GGX (70%) / Lambert materials, "
            "sun + constant environment, 1920x1080, GiTracer maxdepth 8 with Russian roulette after bounce 3, "
            "8 camera samples per pixel per step (one render call; the 256-spp image in 32 steps)")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    return 6650.0, "fallback 6.65 TB/s"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active"

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 4:
                self.samples.append((time.perf_counter(), parts))

    def window(self, t0, t1):
        """Keep only the samples taken inside [t0, t1] (the timed region)."""
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        self.samples = inside if inside else self.samples[-1:]

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        names = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
                 0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
                 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}
        sm, mx, reasons = [], None, set()
        for _, s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                bits = int(s[3], 16) if s[3].startswith("0x") else int(s[3])
                for b, n in names.items():
                    if bits & b and n != "gpu_idle":
                        reasons.add(n)
            except ValueError:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_reference(scene, seconds, rows_per_call=8, nthreads=0, warm=True):
    """Banshee's own CPU tracer (oracle/_ref) on a bounded sample of the frame."""
    from oracle.oracle import Reference
    ncores = os.cpu_count() or 1
    ref = Reference(scene)
    acc = np.zeros((HEIGHT, WIDTH, 4), dtype=np.float32)
    y = 0
    if warm:
        ref.render(spp=1, seed=SEED, maxdepth=MAXDEPTH, region=(0, 0, WIDTH, 1), accum=acc, nthreads=nthreads)
    t0 = time.perf_counter()
    samples = 0
    while time.perf_counter() - t0 < seconds:
        y0 = (y * 131) % (HEIGHT - rows_per_call)
        ref.render(spp=1, seed=SEED, maxdepth=MAXDEPTH, region=(0, y0, WIDTH, y0 + rows_per_call), accum=acc,
                   nthreads=nthreads)
        samples += WIDTH * rows_per_call
        y += 1
    dt = time.perf_counter() - t0
    ref.close()
    return samples / dt / 1e6, dt, samples, (nthreads or ncores), acc


def c3_rows_parity(gs, cpu_acc):
    """relMSE of the GPU's 1-spp frame (sample 0 of every pixel, the same keyed
    samples) against the rows the reference CPU tracer rendered for the CPU
    baseline (a row it rendered k times holds k copies of sample 0)."""
    import torch
    from banshee_b200.metrics import mean_image, relmse
    rows = np.nonzero(cpu_acc[:, 0, 3] > 0)[0]
    frame = torch.zeros((HEIGHT, WIDTH, 4), dtype=torch.float32, device="cuda")
    gs.render(frame.data_ptr(), WIDTH, HEIGHT, 1, seed=SEED, sample_offset=0, maxdepth=MAXDEPTH, stats=False)
    torch.cuda.synchronize()
    got = frame.cpu().numpy()[rows]
    want = cpu_acc[rows]
    return {"rows": int(rows.size), "pixels": int(rows.size * WIDTH),
            "relmse": float(relmse(mean_image(got), mean_image(want))),
            "counts_ok": bool((want[..., 3] == want[:, :1, 3]).all() and (got[..., 3] == 1).all()),
            "error_flags": gs.error_flags(),
            "what": "GPU 1-spp frame vs Banshee's own CPU tracer (oracle/_ref) on the CPU-baseline rows, same keyed samples"}


def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    from banshee_b200 import scenes
    from oracle.oracle import Reference
    sc = scenes.production(WIDTH, HEIGHT)
    ncores = os.cpu_count() or 1
    rows = max(1, min(64, args.ref_rows))
    ref = Reference(sc)
    acc = np.zeros((HEIGHT, WIDTH, 4), dtype=np.float32)

    def step(i):
        y0 = (i * 131) % (HEIGHT - rows)
        ref.render(spp=1, seed=SEED, maxdepth=MAXDEPTH, region=(0, y0, WIDTH, y0 + rows), accum=acc, nthreads=0)

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(args.warmup + i)
    dt = time.perf_counter() - t0
    samples = args.steps * rows * WIDTH
    value = samples / dt / 1e6
    sample = "%d rows x %d px x 1 spp per step (%d camera samples), rows spread over the frame" % (rows, WIDTH, rows * WIDTH)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "sample": sample, "threads": ncores,
                   "implementation": "Banshee GiTracer + Bvh + Mesh compiled unmodified (oracle/_ref), host cores"},
        "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": ncores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def raycast_c2(ctx, nrays=1 << 24, reps=5):
    """C2: 1M-triangle soup, 16M rays per set (coherent 4096^2 pinhole / incoherent),
    closest hit (tmax = FLT_MAX) and any hit (tmax U[0,1]); device-resident rays,
    CUDA-event timing; bytes/ray from an instrumented replay of every 64th ray."""
    import torch
    from banshee_b200 import capi, scenes
    gs = capi.GpuScene(ctx, scenes.soup(1 << 20, seed=1))
    info = gs.info()
    out = {"triangles": info["ntriangles"], "rays_per_set": nrays, "build_ms": info["build_ms"]}
    # the config's four sets, plus coherent shadow rays whose interval ends
    # inside the soup: the config's coherent any-hit set (tmax U[0,1] from 1.5
    # units in front of the cube) is culled at the root and does no work
    sets = [("coherent", False, None), ("coherent", True, None), ("incoherent", False, None),
            ("incoherent", True, None), ("coherent", True, (1.5, 2.5))]
    out["coherent_any_note"] = ("degenerate by construction: rays start 1.5 units in front of the cube and end "
                                "within 1 unit, so every ray is culled at the root (1 node, 0 triangles); "
                                "coherent_shadow_any uses tmax U[1.5,2.5], ending inside the soup")
    for width, (kind, anyhit, trange) in [(w, st) for w in (4, 8) for st in sets]:
        gs.set_node_width(width)
        info = gs.info()
        lay = out.setdefault("layout%d" % width, {"node_width": width, "bvh_nodes": info["nnodes"],
                                                   "node_bytes": info["node_stride"]})
        rays = scenes.soup_rays(nrays, kind, seed=2, any_hit=anyhit, **({"tmax_range": trange} if trange else {}))
        dr = torch.from_numpy(rays.view(np.uint8)).cuda()
        res = torch.zeros(nrays * (1 if anyhit else 16), dtype=torch.uint8, device="cuda")
        fn = gs.intersect_any if anyhit else gs.intersect_closest
        for _ in range(2):
            fn(dr.data_ptr(), res.data_ptr(), nrays)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn(dr.data_ptr(), res.data_ptr(), nrays)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        sub = torch.from_numpy(np.ascontiguousarray(rays[::64]).view(np.uint8)).cuda()
        nodes, tris = gs.traversal_counts(sub.data_ptr(), sub.numel() // 32, anyhit)
        nsub = sub.numel() // 32
        bpr = 32 + (1 if anyhit else 16) + info["node_stride"] * nodes / nsub + 48 * tris / nsub
        name = ("coherent_shadow" if trange else kind) + ("_any" if anyhit else "_closest")
        lay[name] = {
            "mrays_per_s": round(nrays / ms / 1e3, 1), "ms": round(ms, 3), "nodes_per_ray": round(nodes / nsub, 2),
            "tris_per_ray": round(tris / nsub, 2), "bytes_per_ray": round(bpr, 1),
            "achieved_gbs": round(bpr * nrays / (ms * 1e-3) / 1e9, 1)}
        del dr, res, sub
    gs.close()
    out["cpu_baseline"] = _raycast_c2_cpu(scenes.soup(1 << 20, seed=1), nrays)
    # the device builders (LBVH: Morton order; PLOC: clustering over it) on the
    # same soup: build time and traversal speed of their trees
    for builder, name in ((1, "device_lbvh"), (2, "device_ploc"), (3, "device_sah")):
        out[name] = _device_build_traversal(ctx, builder, nrays, reps)
    out["watertight"] = _watertight_traversal(ctx, nrays, reps)
    return out


def _raycast_c2_cpu(sc, nrays, sub=1 << 18, count_sub=1 << 14):
    """C2 on the host: Banshee's own Bvh (oracle/_ref, World::Intersect) casting
    a seeded subset (every nrays/sub-th ray) of each set with all host threads,
    and, as the guard on the byte model, the nodes and triangles per ray of the
    reference's binary tree (the oracle's restatement of Bvh::Build and
    Bvh::Intersect, the same tree) on a smaller subset."""
    try:
        from oracle.oracle import Oracle, Reference
        t0 = time.perf_counter()
        ref = Reference(sc, raycast=True)
        build_s = time.perf_counter() - t0
        orc = Oracle(sc)
    except Exception as exc:   # the checker libraries may be absent
        return {"unavailable": str(exc)}
    from banshee_b200 import scenes
    out = {"kind": "reference", "cores": os.cpu_count() or 1, "reference_build_s": build_s,
           "sample": "every %dth ray of each 16M-ray set (%d rays), all host threads" % (nrays // sub, sub)}
    for kind, anyhit, trange in [("coherent", False, None), ("incoherent", False, None),
                                 ("incoherent", True, None), ("coherent", True, (1.5, 2.5))]:
        rays = scenes.soup_rays(nrays, kind, seed=2, any_hit=anyhit, **({"tmax_range": trange} if trange else {}))
        r = np.ascontiguousarray(rays[:: nrays // sub])
        t0 = time.perf_counter()
        (ref.intersect_any if anyhit else ref.intersect_closest)(r, nthreads=0)
        dt = time.perf_counter() - t0
        c = np.ascontiguousarray(rays[:: nrays // count_sub])
        nodes, tris = orc.traversal_counts(c, any_hit=anyhit)
        name = ("coherent_shadow" if trange else kind) + ("_any" if anyhit else "_closest")
        out[name] = {"mrays_per_s": round(r.shape[0] / dt / 1e6, 3),
                     "reference_nodes_per_ray": round(nodes / c.shape[0], 2),
                     "reference_tris_per_ray": round(tris / c.shape[0], 2)}
    ref.close()
    orc.close()
    return out


def _watertight_traversal(ctx, nrays, reps):
    """The optional watertight ray / triangle test (not in the reference) on the
    same soup and rays, host SAH tree: Mrays/s per set and node layout."""
    import torch
    from banshee_b200 import abi, capi, scenes
    gw = capi.GpuScene(ctx, scenes.soup(1 << 20, seed=1), intersect=abi.BG_INTERSECT_WATERTIGHT)
    res = {}
    for kind, anyhit in (("coherent", False), ("incoherent", False), ("incoherent", True)):
        rays = scenes.soup_rays(nrays, kind, seed=2, any_hit=anyhit)
        dr = torch.from_numpy(rays.view(np.uint8)).cuda()
        out = torch.zeros(nrays * (1 if anyhit else 16), dtype=torch.uint8, device="cuda")
        fn = gw.intersect_any if anyhit else gw.intersect_closest
        for width in (4, 8):
            gw.set_node_width(width)
            for _ in range(2):
                fn(dr.data_ptr(), out.data_ptr(), nrays)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn(dr.data_ptr(), out.data_ptr(), nrays)
            e1.record()
            torch.cuda.synchronize()
            res["layout%d_%s_%s_mrays_per_s" % (width, kind, "any" if anyhit else "closest")] = round(
                nrays / (e0.elapsed_time(e1) / reps) / 1e3, 1)
        del dr, out
    gw.close()
    return res


def _device_build_traversal(ctx, builder, nrays, reps):
    import torch
    from banshee_b200 import capi, scenes
    t0 = time.perf_counter()
    gl = capi.GpuScene(ctx, scenes.soup(1 << 20, seed=1), builder=builder)
    lb = {"build_ms": gl.info()["build_ms"], "build_wall_s": time.perf_counter() - t0}
    for width in (4, 8):
        gl.set_node_width(width)
        for kind in ("coherent", "incoherent"):
            rays = scenes.soup_rays(nrays, kind, seed=2)
            dr = torch.from_numpy(rays.view(np.uint8)).cuda()
            res = torch.zeros(nrays * 16, dtype=torch.uint8, device="cuda")
            for _ in range(2):
                gl.intersect_closest(dr.data_ptr(), res.data_ptr(), nrays)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                gl.intersect_closest(dr.data_ptr(), res.data_ptr(), nrays)
            e1.record()
            torch.cuda.synchronize()
            lb["layout%d_%s_closest_mrays_per_s" % (width, kind)] = nrays / (e0.elapsed_time(e1) / reps) / 1e3
            del dr, res
    gl.close()
    return lb


def cornell_c1(ctx, ref_seconds_cap=60.0):
    """C1: Cornell box 256x256, 64 spp, GiTracer(5): GPU Msamples/s and relMSE of the
    GPU image against Banshee's own CPU render of the same samples (oracle/_ref)."""
    import torch
    from banshee_b200 import capi, scenes
    from banshee_b200.metrics import mean_image, relmse
    sc = scenes.cornell(256, 256)
    gs = capi.GpuScene(ctx, sc)
    acc = torch.zeros((256, 256, 4), dtype=torch.float32, device="cuda")
    # pass size and block size picked for the whole 64-spp render (it is one call)
    tune = gs.autotune(acc.data_ptr(), 256, 256, probe_spp=64, maxdepth=5)
    gs.render(acc.data_ptr(), 256, 256, 64, seed=1, maxdepth=5, stats=False)
    acc.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    gs.render(acc.data_ptr(), 256, 256, 64, seed=1, maxdepth=5, stats=False)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"resolution": [256, 256], "spp": 64, "maxdepth": 5, "gpu_ms": ms, "gpu_msamples_per_s": 256 * 256 * 64 / ms / 1e3,
           "autotune": tune}
    try:
        from oracle.oracle import Reference
        t0 = time.perf_counter()
        ref = Reference(sc).render(spp=64, seed=1, maxdepth=5)
        dt = time.perf_counter() - t0
        out.update({"reference_cpu_s": dt, "reference_cpu_msamples_per_s": 256 * 256 * 64 / dt / 1e6,
                    "reference_cores": os.cpu_count(),
                    "relmse_gpu_vs_reference": relmse(mean_image(acc.cpu().numpy()), mean_image(ref))})
    except Exception as exc:
        out["reference"] = "unavailable: %s" % exc
    gs.close()
    return out


def batch_c4(ctx, nscenes=64, seed=7, timed_frames=1, rank=0, world=1, dist=None, builders=((3, "device_sah"),)):
    """C4: 64 procedural scenes (triangles log-uniform in [1e4, 5e5], resolutions from
    {256^2, 512^2, 1024x768}, 16..128 spp each) traced together by one batch: one set of
    queues, persistent kernels, one pass graph; autotuned node width / block / wavefront
    sizes.  Each builder in `builders` (default: the device binned SAH; --c4-all-builders
    adds host binned SAH, device LBVH and PLOC) builds the scenes (wall time, scene
    generation excluded) and the batch renders its trees; the headline fields are the first
    builder's row.  On N GPUs each rank takes every N-th scene (no exchange); times are the
    max over ranks."""
    import torch
    from banshee_b200 import capi, multigpu, scenes
    t0 = time.perf_counter()
    all_items = scenes.batch(nscenes, seed=seed)
    gen_s = time.perf_counter() - t0
    items = multigpu.shard(all_items, rank, world)
    bufs, jobs = [], []
    for k, (sc, spp) in enumerate(items):
        acc = torch.zeros((sc.height, sc.width, 4), dtype=torch.float32, device="cuda")
        bufs.append(acc)
        jobs.append(dict(scene=k, width=sc.width, height=sc.height, spp=spp, seed=1, camera=sc.camera_desc(),
                         accum_dev=acc.data_ptr()))
    samples = sum(sc.width * sc.height * spp for sc, spp in all_items)
    rows = {}
    for builder, name in builders:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        gss = [capi.GpuScene(ctx, sc, builder=builder) for sc, _ in items]
        batch = capi.Batch(ctx, gss)
        torch.cuda.synchronize()
        build_s = multigpu.max_over_ranks(time.perf_counter() - t1, dist, device="cuda")
        for g in gss:
            g.close()
        tune = batch.autotune(jobs, probe_spp=2, maxdepth=MAXDEPTH)
        for b in bufs:
            b.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(timed_frames):
            batch.render(jobs, maxdepth=MAXDEPTH)
        e1.record()
        torch.cuda.synchronize()
        ms = multigpu.max_over_ranks(e0.elapsed_time(e1) / timed_frames, dist, device="cuda")
        info = batch.info()
        batch.close()
        rows[name] = {"build_s": build_s, "ms": ms, "msamples_per_s": samples / ms / 1e3,
                      "build_plus_frame_s": build_s + ms / 1e3, "node_width": info["node_width"], "autotune": tune}
    head = rows[builders[0][1]]
    return {"scenes": nscenes, "triangles_total": sum(sc.ntriangles for sc, _ in all_items),
            "camera_samples": samples, "scenes_per_rank": len(items), "builder": builders[0][1],
            "node_width": head["node_width"],
            "ms": head["ms"], "msamples_per_s": head["msamples_per_s"], "autotune": head["autotune"],
            "build_s": head["build_s"], "scene_generation_s": gen_s, "by_builder": rows,
            "resolutions": sorted({"%dx%d" % (sc.width, sc.height) for sc, _ in all_items}),
            "spp_range": [min(s for _, s in all_items), max(s for _, s in all_items)],
            "triangle_range": [min(sc.ntriangles for sc, _ in all_items),
                               max(sc.ntriangles for sc, _ in all_items)]}


def _ground_truth(gs, args, maxdepth, spp, camera=None, width=WIDTH, height=HEIGHT, name="c3"):
    """Plain GiTracer(maxdepth) render of the full frame at `spp` samples per pixel,
    float64 accumulation of 256-spp chunks, checkpointed under --gt-cache (resumed
    when the same reference was started before).  Returns (mean, variance of the
    mean, seconds of this run, spp resumed from a checkpoint)."""
    from banshee_b200 import groundtruth as GT
    key = {"scene": name, "w": width, "h": height, "maxdepth": maxdepth, "seed": 7777, "spp": spp,
           "triangles": gs.info()["ntriangles"]}
    path = None
    if args.gt_cache:
        os.makedirs(args.gt_cache, exist_ok=True)
        path = os.path.join(args.gt_cache, "gt_%s_d%d_%d.npz" % (name, maxdepth, spp))
    start = {}
    t0 = time.perf_counter()

    def chunk(acc32, off, n):
        start.setdefault("spp", off)
        gs.render(acc32.data_ptr(), width, height, n, seed=7777, sample_offset=off, maxdepth=maxdepth, camera=camera,
                  stats=False)

    acc = GT.accumulate(chunk, height, width, spp, key, chunk=256, path=path, every=32)
    import torch
    torch.cuda.synchronize()
    return acc.mean(), acc.mean_variance(), time.perf_counter() - t0, start.get("spp", spp)


def _summ(r):
    return {"seconds_to_target": r["t_target"], "frames": r["frames"], "final_relmse": r["final_relmse"],
            "ms_per_frame": 1e3 * r["seconds"] / max(1, r["frames"]),
            "curve": [[round(t, 4), n, float("%.4g" % e)] for t, n, e in r["curve"][::max(1, len(r["curve"]) // 12)]]}


C5_REPEATS = 3


def _median_run(runs):
    """The run with the median time to the target (a run that never reached it counts as the slowest)."""
    order = sorted(runs, key=lambda r: r["t_target"] if r["t_target"] is not None else float("inf"))
    return order[len(order) // 2]


def _ratio(a, b):
    return (a / b) if (a and b) else None


WARM_FRAMES, WARM_W, WARM_H = 32, 384, 216   # the cache's training-only warm-up frames
CACHE_CFG = dict(log2_table_size=19, base_resolution=16, max_resolution=2048, train_paths=65536, cache_depth=2,
                 train_batch=65536, train_steps=1, learning_rate=1e-2, train_suffix=1)
CACHE_DESC = ("hash grid 16 levels x 2 features, 2^19 entries/level, res 16..2048; MLP 64x5 bf16; Adam lr 1e-2; "
              "65536 training paths/frame; rendering paths end into the cache after 2 bounces, training paths one "
              "bounce later (self-training); one Adam step per frame over up to 65536 training vertices from depth 2 "
              "on, trained one frame behind beside the next frame's first bounces")


def time_to_relmse(gs, sc, args, target=1e-3):
    """Second half of the metric, on the full 1920x1080 frame: GPU time for the
    radiance-cache tracer and for the plain tracer to reach relMSE 1e-3 against a
    plain GiTracer(8) render at args.gt_spp spp accumulated in float64 (the
    reference's own noise, estimated from two halves, subtracted).  The plain
    tracer runs at 1 spp per frame and at SPP per call (its throughput
    configuration, the headline comparison, timed C5_REPEATS times like the
    cache's, medians compared); the cache renders SPP per frame
    after 32 training-only frames (every path of a 384x216 frame trains; their
    time counts) and trains once per frame; it is also timed at 1 spp per frame
    against the plain tracer at 1 spp per frame.  The cache's bias floor is its error, after
    convergence, once its image noise and the reference's are taken out.  The
    bound for any cache that ends paths after 2 bounces is the plain tracer
    truncated there (max depth 2) against its own float64 reference."""
    import torch
    from banshee_b200 import capi
    from banshee_b200 import convergence as CV
    gt, gt_var, gt_s, gt_from = _ground_truth(gs, args, MAXDEPTH, args.gt_spp)
    run = lambda fn, every: CV.converge_frame(fn, WIDTH, HEIGHT, gt, gt_var, args.conv_seconds, 100000,
                                              target=target, every=every)
    plain = run(lambda p, f: gs.render(p, WIDTH, HEIGHT, 1, seed=SEED, sample_offset=f, maxdepth=MAXDEPTH,
                                       stats=False), 4)
    # the two tracers at their throughput configurations (the headline ratio) are
    # timed C5_REPEATS times each, the cache from a fresh, untrained cache every
    # time; the medians are compared
    plain_spp_runs = [run(lambda p, f: gs.render(p, WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=f * SPP,
                                                 maxdepth=MAXDEPTH, stats=False), 1) for _ in range(C5_REPEATS)]
    plain_spp = _median_run(plain_spp_runs)
    # warm the process as the plain tracer's timing is warm (its pass graph was
    # captured by the steps above): a throwaway cache of the same configuration
    # renders two frames of each shape the timed caches render (kernel modules
    # loaded, scratch memory pooled, pass graphs captured for both training-row
    # sets); the timed caches then start untrained
    warm = capi.RadianceCache(gs, **CACHE_CFG)
    wbuf = torch.zeros((HEIGHT, WIDTH, 4), dtype=torch.float32, device="cuda")
    wscr = torch.zeros((WARM_H, WARM_W, 4), dtype=torch.float32, device="cuda")
    for f in range(2):
        warm.render(wbuf.data_ptr(), WIDTH, HEIGHT, 1, seed=SEED, sample_offset=f, maxdepth=MAXDEPTH)
    for f in range(2):
        warm.render(wscr.data_ptr(), WARM_W, WARM_H, 1, seed=SEED, sample_offset=f, maxdepth=MAXDEPTH)
    for f in range(2):
        warm.render(wbuf.data_ptr(), WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=f * SPP, maxdepth=MAXDEPTH)
    torch.cuda.synchronize()
    del wbuf, wscr
    # the cache at 1 spp per frame (one Adam step per frame)
    cache1 = capi.RadianceCache(gs, **CACHE_CFG)
    cached1 = run(lambda p, f: cache1.render(p, WIDTH, HEIGHT, 1, seed=SEED, sample_offset=f, maxdepth=MAXDEPTH), 4)
    # the cache at its throughput configuration: WARM_FRAMES training-only frames
    # (the same camera at 384x216, 1 spp: every path is a training path, nothing
    # is kept), then SPP samples per pixel per frame; the warm-up is timed
    scratch = torch.zeros((WARM_H, WARM_W, 4), dtype=torch.float32, device="cuda")
    caches, cached_runs = [], []
    for _ in range(C5_REPEATS):
        cache = capi.RadianceCache(gs, **CACHE_CFG)
        caches.append(cache)

        def render_cached(p, f, cache=cache):
            if f < WARM_FRAMES:
                cache.render(scratch.data_ptr(), WARM_W, WARM_H, 1, seed=SEED + 99, sample_offset=f,
                             maxdepth=MAXDEPTH)
            else:
                cache.render(p, WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=(f - WARM_FRAMES) * SPP,
                             maxdepth=MAXDEPTH)

        cached_runs.append(run(render_cached, 1))
    cached = _median_run(cached_runs)
    cache = caches[cached_runs.index(cached)]
    # the median run's cache keeps training while the floor is measured
    floor = CV.bias_floor(lambda p, f: cache.render(p, WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=f * SPP,
                                                    maxdepth=MAXDEPTH),
                          WIDTH, HEIGHT, gt, gt_var, args.floor_frames, first_frame=cached["frames"])
    # the caches are released after every timed leg that uses one (a release
    # synchronises the device and frees about 0.6 GB)
    for c in [warm, cache1] + caches:
        c.close()
    del scratch
    gt2, gt2_var, gt2_s, _ = _ground_truth(gs, args, 2, args.gt_spp_bound)
    trunc = CV.converge_frame(lambda p, f: gs.render(p, WIDTH, HEIGHT, 1, seed=SEED, sample_offset=f, maxdepth=2,
                                                     stats=False),
                              WIDTH, HEIGHT, gt2, gt2_var, args.conv_seconds, 100000, target=target, every=4)
    del gt, gt_var, gt2, gt2_var
    ratio = _ratio(cached1["t_target"], plain["t_target"])
    ratio_spp = _ratio(cached["t_target"], plain_spp["t_target"])
    bound = _ratio(trunc["t_target"], plain["t_target"])
    return {"target_relmse": target, "frame": [WIDTH, HEIGHT], "reference_spp": args.gt_spp,
            "reference_seconds": gt_s, "reference_resumed_from_spp": gt_from,
            "reference": "plain GiTracer(8), full frame, float64 accumulation of 256-spp chunks in two halves",
            "relmse": "mean over pixels and channels of (x - ref)^2 / (ref^2 + 0.01), minus the same mean of the "
                      "reference's own variance (from its two halves)",
            "cache_config": CACHE_DESC,
            "plain": _summ(plain),
            "plain_spp_per_call": {"spp_per_call": SPP, "seconds_to_target_runs": [r["t_target"] for r in plain_spp_runs],
                                   **_summ(plain_spp)},
            "cache": {"spp_per_frame": SPP, "warm_up_frames": [WARM_FRAMES, WARM_W, WARM_H],
                      "seconds_to_target_runs": [r["t_target"] for r in cached_runs], **_summ(cached)},
            "cache_1spp": _summ(cached1), "cache_bias_floor": floor,
            "cache_over_plain_time": ratio_spp, "cache_1spp_over_plain_1spp_time": ratio,
            "perfect_cache_bound": {
                "what": "plain tracer truncated after 2 bounces (max depth 2) against its own reference at "
                        "%d spp: the time-to-target of a free, exact cache ending paths there" % args.gt_spp_bound,
                "reference_seconds": gt2_s, **_summ(trunc), "over_plain_time": bound},
            "summary_cache_over_plain_best": ratio_spp, "summary_cache_over_plain_1spp": ratio,
            "summary_bias_floor": floor["bias_floor"], "summary_truncation_bound": bound,
            "summary_reference_spp": args.gt_spp}


def cache_bias_scenes(ctx, args, warm_frames=64):
    """The cache's bias floor on two more scenes than C5's: the C1 Cornell box
    (256^2, GiTracer(5): an indoor scene whose light comes from paths of many
    bounces) and a reduced production scene (512^2, 200k-triangle terrain and
    20 spheres, GiTracer(8)).  Same cache configuration and measurement as
    C5: after `warm_frames` training frames at SPP per frame, the relMSE of
    args.floor_frames more frames against a plain render at args.gt_spp_bound
    spp accumulated in float64, split into the image's noise, the reference's
    noise and the rest, the squared bias.  Also with the training paths traced
    to full depth instead of ending into the cache (unbiased training targets:
    what remains is the network's and the grid's fitting error)."""
    from banshee_b200 import capi, scenes
    from banshee_b200 import convergence as CV
    out = []
    for name, sc, maxdepth in (("cornell_c1", scenes.cornell(256, 256), 5),
                               ("production_512", scenes.production(512, 512, nterrain=320, nspheres=20,
                                                                    sphere_seg=60, seed=11), MAXDEPTH)):
        gs = capi.GpuScene(ctx, sc)
        W, H = sc.width, sc.height
        gt, gt_var, gt_s, _ = _ground_truth(gs, args, maxdepth, args.gt_spp_bound, width=W, height=H, name=name)
        import torch
        tmp = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        rec = {"scene": name, "frame": [W, H], "maxdepth": maxdepth, "triangles": gs.info()["ntriangles"],
               "reference_spp": args.gt_spp_bound, "reference_seconds": gt_s, "warm_frames": warm_frames}
        # the C5 configuration (training paths end into the cache one bounce after
        # the rendering paths), and training paths traced to full depth
        for key, cfg in (("", CACHE_CFG), ("full_depth_training_", dict(CACHE_CFG, train_suffix=0))):
            cache = capi.RadianceCache(gs, **cfg)
            for f in range(warm_frames):
                cache.render(tmp.data_ptr(), W, H, SPP, seed=SEED, sample_offset=f * SPP, maxdepth=maxdepth)
            floor = CV.bias_floor(lambda p, f: cache.render(p, W, H, SPP, seed=SEED, sample_offset=f * SPP,
                                                            maxdepth=maxdepth),
                                  W, H, gt, gt_var, args.floor_frames, first_frame=warm_frames)
            torch.cuda.synchronize()
            cache.close()
            rec.update({key + k: v for k, v in floor.items()})
        out.append(rec)
        del gt, gt_var, tmp
        gs.close()
    return out


def summary(line):
    """A few numbers per config, kept short so the end of the JSON line carries them."""
    def g(d, *ks):
        for k in ks:
            if not isinstance(d, dict) or d.get(k) is None:
                return None
            d = d[k]
        return float("%.6g" % d) if isinstance(d, float) else d
    out = {"c3_msamples_per_s": g(line, "value"), "c3_e2e_msamples_per_s": g(line, "e2e", "value"),
           "c3_parity_relmse": g(line, "c3_parity", "relmse"), "c3_parity_pixels": g(line, "c3_parity", "pixels"),
           "traversal_frac_hbm": g(line, "roofline", "frac"), "error_flags": line.get("error_flags")}
    c2 = line.get("raycast_c2")
    if c2:
        for w in (4, 8):
            for k in ("coherent_closest", "incoherent_closest", "incoherent_any", "coherent_shadow_any"):
                out["c2_w%d_%s_mrays" % (w, k)] = g(c2, "layout%d" % w, k, "mrays_per_s")
    out["c2_watertight_w4_incoherent_closest_mrays"] = g(line, "raycast_c2", "watertight",
                                                        "layout4_incoherent_closest_mrays_per_s")
    out["c2_cpu_reference_incoherent_closest_mrays"] = g(line, "raycast_c2", "cpu_baseline", "incoherent_closest",
                                                         "mrays_per_s")
    out["c1_msamples_per_s"] = g(line, "cornell_c1", "gpu_msamples_per_s")
    out["c1_relmse_vs_reference"] = g(line, "cornell_c1", "relmse_gpu_vs_reference")
    out["c4_msamples_per_s"] = g(line, "batch_c4", "msamples_per_s")
    out["c4_autotune"] = [g(line, "batch_c4", "autotune", k) for k in ("node_width", "trace_threads", "paths_per_pass")]
    rt = line.get("relmse_time")
    if rt:
        for k, v in rt.items():
            if k.startswith("summary_"):
                out["c5_" + k[len("summary_"):]] = v
        for r in rt.get("bias_per_scene") or []:
            out["c5_bias_floor_" + r["scene"]] = g(r, "bias_floor")
            out["c5_bias_floor_full_depth_training_" + r["scene"]] = g(r, "full_depth_training_bias_floor")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU-baseline sample (seconds)")
    ap.add_argument("--ref-rows", type=int, default=8, help="rows per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cache", action="store_true", help="skip the time-to-relMSE measurement")
    ap.add_argument("--no-extra", action="store_true", help="skip the C1 / C2 sections")
    ap.add_argument("--no-c4", action="store_true", help="skip the 64-scene batch (C4)")
    ap.add_argument("--c4-all-builders", action="store_true", help="C4 with every BVH builder, not only device SAH")
    ap.add_argument("--gt-spp", type=int, default=65536, help="spp of the float64 reference frame")
    ap.add_argument("--gt-spp-bound", type=int, default=16384, help="spp of the depth-2 reference (the bound)")
    ap.add_argument("--gt-cache", default=None, help="directory for reference checkpoints (resumed when present)")
    ap.add_argument("--floor-frames", type=int, default=256, help="cache frames of the bias-floor measurement")
    ap.add_argument("--conv-seconds", type=float, default=20.0, help="time budget per tracer for time-to-relMSE")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    from banshee_b200 import abi, capi, multigpu, scenes

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        dist = multigpu.init("nccl", timeout_s=120, device=torch.device("cuda", local))

    t_scene = time.perf_counter()
    sc = scenes.production(WIDTH, HEIGHT)
    ctx = capi.Context(local)
    gs = capi.GpuScene(ctx, sc)
    info = gs.info()
    t_scene = time.perf_counter() - t_scene
    stream = torch.cuda.current_stream()
    acc = torch.zeros((HEIGHT, WIDTH, 4), dtype=torch.float32, device="cuda")
    npix = WIDTH * HEIGHT
    # the framework's autotuner picks node layout, traversal block size and paths per pass
    tune = gs.autotune(acc.data_ptr(), WIDTH, HEIGHT, probe_spp=SPP, maxdepth=MAXDEPTH, stream=stream.cuda_stream)
    acc.zero_()
    info = gs.info()

    # N = 1: steps render straight into acc.  N > 1: each step renders this
    # rank's samples into a zeroed step buffer, one all-reduce sums the ranks'
    # step buffers and the sum is added once into acc
    frame = multigpu.StepExchange(acc, dist)

    def step(i, stats=False, flags=0):
        return gs.render(frame.target.data_ptr(), WIDTH, HEIGHT, SPP, seed=SEED,
                         sample_offset=multigpu.sample_offset(i, rank, world, SPP), tracer=abi.BG_TRACER_GI,
                         maxdepth=MAXDEPTH, stream=stream.cuda_stream, flags=flags, stats=stats)

    def exchange():
        frame.end_step()

    # warm-up (untimed)
    for i in range(args.warmup):
        step(i)
        exchange()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    torch.cuda.nvtx.range_push("timed_steps")   # lets a profiler select the timed launches
    for i in range(args.steps):
        step(args.warmup + i)
        exchange()
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    w1 = time.perf_counter()
    if dist is not None:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    time.sleep(0.25)
    clocks.stop()
    clocks.window(w0, w1 + 0.05)
    ms = multigpu.max_over_ranks(ms, dist, device="cuda")
    samples_total = world * npix * SPP * args.steps
    value = samples_total / (ms * 1e-3) / 1e6
    flags_err = gs.error_flags()

    # one instrumented step: per-phase CUDA-event timing + 1/64 traversal replay
    st = step(args.warmup + args.steps, stats=True, flags=abi.BG_RENDER_TIME_PHASES | abi.BG_RENDER_COUNT_TRAVERSAL)
    st_plain = step(args.warmup + args.steps + 1, stats=True, flags=abi.BG_RENDER_TIME_PHASES)
    launches_per_step = st_plain["kernel_launches"]
    node_b = info["node_stride"]
    tri_b = 48
    nodes_per_ray = st["sub_nodes_extension"] / max(1, st["sub_rays_extension"])
    tris_per_ray = st["sub_tris_extension"] / max(1, st["sub_rays_extension"])
    bytes_per_ray = 32 + 16 + node_b * nodes_per_ray + tri_b * tris_per_ray
    ext_rays = st_plain["rays_extension"]
    ext_bytes = ext_rays * bytes_per_ray
    ext_ms = st_plain["ms_extend"]
    achieved = ext_bytes / (ext_ms * 1e-3) / 1e9
    peak, peak_src = peaks()
    traffic = None
    measured = {}
    prof = os.path.join(ROOT, "profiles", "traverse_extend_c3.json")
    if os.path.exists(prof):
        with open(prof) as f:
            p = json.load(f)
        if "dram_bytes_per_ray" in p:
            traffic = p["dram_bytes_per_ray"] * ext_rays / max(1, st_plain["launches_extend"])
        # what the kernel really moves (ncu, one 1-spp frame, scaled by rays): the
        # byte model above counts node and triangle bytes wherever they are served
        # from; DRAM and L2 bytes and SIMT efficiency say where the time goes
        for k in ("dram_bytes_per_ray", "l2_bytes_per_ray", "l2_pct_of_peak", "threads_per_instruction",
                  "dram_pct_of_peak", "sm_pct_of_peak"):
            if k in p:
                measured[k] = p[k]
    roofline = {
        "kernel": "k_trace<closest> on the extension-ray queues (all bounces of one step)",
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "peak_source": peak_src,
        "traffic": traffic,
        "algorithmic_bytes_per_launch": ext_bytes / max(1, st_plain["launches_extend"]),
        "bytes_per_ray": bytes_per_ray, "nodes_per_ray": nodes_per_ray, "tris_per_ray": tris_per_ray,
        "node_bytes": node_b, "tri_bytes": tri_b,
        "launches": st_plain["launches_extend"], "ms_extend": ext_ms, "ms_step": st_plain["ms_total"],
        "byte_model": "32 B ray + 16 B hit + node_bytes * nodes/ray + 48 B * triangles/ray, counts from an "
                      "instrumented replay of every 64th ray of each extension queue; frac counts those bytes "
                      "wherever they are served from (mostly L1/L2), see ncu_measured",
        "ncu_measured": measured or None,
    }
    rays_per_step = st_plain["rays_closest"] + st_plain["rays_any"]
    # every k_trace launch of the step (extension, shadow any-hit, MIS): the
    # traversal kernel's whole share of the step; a shadow ray also reads its
    # slot index and contribution (20 B), a closest-hit ray writes a 16 B hit
    any_rays = st_plain["rays_any"]
    mis_rays = st_plain["rays_closest"] - ext_rays

    def per_ray(kind, extra):
        n = max(1, st["sub_rays_" + kind])
        nodes, tris = st["sub_nodes_" + kind] / n, st["sub_tris_" + kind] / n
        return 32 + extra + node_b * nodes + tri_b * tris, nodes, tris

    any_b, any_nodes, any_tris = per_ray("any", 20)
    mis_b, _, _ = per_ray("mis", 16) if st["sub_rays_mis"] > 0 else (bytes_per_ray, 0, 0)
    all_bytes = ext_bytes + any_rays * any_b + mis_rays * mis_b
    all_ms = st_plain["ms_extend"] + st_plain["ms_shadow"] + st_plain["ms_mis"]
    all_achieved = all_bytes / (all_ms * 1e-3) / 1e9
    roofline_all = {
        "kernel": "k_trace, every launch of one step (extension + shadow any-hit + MIS)",
        "bound": "hbm", "achieved": all_achieved, "peak": peak, "unit": "GB/s", "frac": all_achieved / peak,
        "peak_source": peak_src, "traffic": None,
        "rays": {"extension": ext_rays, "any": any_rays, "mis": mis_rays},
        "bytes_per_any_ray": any_b, "nodes_per_any_ray": any_nodes, "tris_per_any_ray": any_tris,
        "ms": all_ms,
    }

    # e2e through the public host-buffer entry point (pinned host accumulation buffer)
    host = torch.zeros((HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()
    ek = max(3, min(args.steps, 10))
    for i in range(2):
        gs.render_host(WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=i * SPP, maxdepth=MAXDEPTH, accum=host_np)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(ek):
        gs.render_host(WIDTH, HEIGHT, SPP, seed=SEED, sample_offset=multigpu.sample_offset(2 + i, rank, world, SPP),
                       maxdepth=MAXDEPTH, accum=host_np)
    e2e_s = time.perf_counter() - t0
    e2e_s = multigpu.max_over_ranks(e2e_s, dist, device="cuda")
    e2e_value = world * npix * SPP * ek / e2e_s / 1e6

    cpu = None
    c3_parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, dt, n, cores, cpu_acc = cpu_baseline_reference(sc, args.cpu_seconds)
            cpu = {"value": v, "unit": "Msamples/s", "cores": cores, "kind": "reference",
                   "sample": "%d camera samples (%d rows x %d px x 1 spp) in %.1f s with %d threads"
                             % (n, n // WIDTH, WIDTH, dt, cores)}
            c3_parity = c3_rows_parity(gs, cpu_acc)
        except Exception as exc:   # the checker library may be absent
            cpu = {"value": None, "unit": "Msamples/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % exc}

    cache_res = c2 = c1 = None
    if rank == 0 and world == 1 and not args.no_cache:
        cache_res = time_to_relmse(gs, sc, args)
        cache_res["bias_per_scene"] = cache_bias_scenes(ctx, args)
        # the reference CPU tracer's time to the same target: the samples the plain
        # GPU tracer needed (same estimator) at the CPU rate measured above
        ps = cache_res["plain_spp_per_call"]
        if cpu and cpu.get("value") and ps.get("seconds_to_target"):
            samples = ps["seconds_to_target"] / (ps["ms_per_frame"] * 1e-3) * SPP * npix
            cache_res["cpu_reference_seconds_to_target"] = samples / (cpu["value"] * 1e6)
            cache_res["summary_cpu_reference_seconds_to_target"] = cache_res["cpu_reference_seconds_to_target"]
    if rank == 0 and world == 1 and not args.no_extra:
        gs.close()
        c2 = raycast_c2(ctx)
        c1 = cornell_c1(ctx)
    c4 = None
    if not args.no_c4:
        blds = (((3, "device_sah"), (0, "host_sah"), (1, "device_lbvh"), (2, "device_ploc")) if args.c4_all_builders
                else ((3, "device_sah"),))
        c4 = batch_c4(ctx, rank=rank, world=world, dist=dist, builders=blds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": WORKLOAD, "triangles": info["ntriangles"], "resolution": [WIDTH, HEIGHT],
                       "spp_per_step": SPP, "maxdepth": MAXDEPTH, "parallelism": "dp%d (samples)" % world,
                       "l2": "inputs larger than L2: scene %.2f GB resident in HBM (126 MB L2)"
                             % ((info["node_bytes"] + info["tri_bytes"] + info["shade_bytes"]) / 1e9),
                       "scene_build_s": t_scene, "autotune": tune},
            "mrays_per_s": world * rays_per_step * args.steps / (ms * 1e-3) / 1e6,
            "rays_per_sample": rays_per_step / (npix * SPP),
            "roofline": roofline,
            "roofline_traversal_all": roofline_all,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": npix * 16,
                    "d2h_bytes_per_step": npix * 16, "api": "bg_render_host (pinned host RGBW buffer)"},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks.summary(),
            "error_flags": flags_err,
            "phase_ms": {"extend": st_plain["ms_extend"], "shadow": st_plain["ms_shadow"],
                         "mis": st_plain["ms_mis"], "shade_and_rest": st_plain["ms_shade"]},
            "raycast_c2": c2,
            "cornell_c1": c1,
            "batch_c4": c4,
            "relmse_time": cache_res,
            "c3_parity": c3_parity,
        }
        line["summary"] = summary(line)     # last key: the short record of every config
        print(json.dumps(line), flush=True)
        print("summary: " + json.dumps(line["summary"]), file=sys.stderr, flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
