"""Multi-process sharding of the path tracer, on CPU with gloo (world size 2).

Each rank renders its share of the samples (sample_offset = (step * N + rank) *
spp) with the CPU oracle standing in for its GPU, the ranks all-reduce their
accumulation buffers, and the result must equal one process rendering every
sample (up to float summation order).  The exchange runs after every step, as
the bench's does, and every pixel's sample count must be exact after each one.  A second test makes one rank leave
before the collective: the other must get an error from the process-group
timeout instead of hanging.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker_render(rank, world, port, steps, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    from banshee_b200 import multigpu, scenes
    from oracle.oracle import Oracle
    dist = multigpu.init("gloo", timeout_s=60)
    sc = scenes.cornell(16, 16)
    o = Oracle(sc)
    total = torch.zeros((16, 16, 4), dtype=torch.float32)
    ex = multigpu.StepExchange(total, dist)
    for step in range(steps):
        # each step renders this rank's samples into the step buffer, then the
        # ranks exchange and the running total grows by that step only
        o.render(spp=1, seed=5, maxdepth=5, sample_offset=multigpu.sample_offset(step, rank, world),
                 accum=ex.target.numpy(), nthreads=1)
        ex.end_step()
        # after step k every pixel holds exactly (k + 1) * world samples
        assert (total[..., 3] == float((step + 1) * world)).all(), (step, total[..., 3].unique())
    ms = multigpu.max_over_ranks(10.0 * (rank + 1), dist)
    if rank == 0:
        np.save(out_path, total.numpy())
        with open(out_path + ".ms", "w") as f:
            f.write(str(ms))
    dist.barrier()
    dist.destroy_process_group()


def _worker_leave(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    from banshee_b200 import multigpu
    dist = multigpu.init("gloo", timeout_s=5)
    if rank == 1:
        os._exit(0)                      # leaves between steps, before the collective
    t = torch.ones(4)
    try:
        multigpu.combine(t, dist)
        msg = "no error"
    except Exception as exc:             # the short process-group timeout ends the collective
        msg = "error: " + type(exc).__name__
    with open(out_path, "w") as f:
        f.write(msg)
    os._exit(0)


def test_sharded_render_equals_single_process(tmp_path, oracle_built):
    import torch.multiprocessing as mp
    from banshee_b200 import scenes
    from oracle.oracle import Oracle
    out = str(tmp_path / "acc.npy")
    world, steps = 2, 4
    mp.start_processes(_worker_render, args=(world, _free_port(), steps, out), nprocs=world, start_method="spawn")
    got = np.load(out)
    ref = Oracle(scenes.cornell(16, 16)).render(spp=world * steps, seed=5, maxdepth=5, nthreads=1)
    assert (got[..., 3] == ref[..., 3]).all()
    np.testing.assert_allclose(got[..., :3], ref[..., :3], rtol=1e-5, atol=1e-6)
    assert float(open(out + ".ms").read()) == 20.0      # max over ranks


def test_rank_leaving_is_reported_not_hung(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "leave.txt")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker_leave, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(not p.is_alive() for p in procs)
    assert open(out).read().startswith("error"), open(out).read()


def test_scene_sharding_covers_every_scene_once():
    from banshee_b200 import multigpu
    items = list(range(64))
    for world in (1, 2, 3, 8):
        parts = [multigpu.shard(items, r, world) for r in range(world)]
        assert sorted(x for p in parts for x in p) == items
        assert max(map(len, parts)) - min(map(len, parts)) <= 1
