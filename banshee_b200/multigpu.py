"""Data-parallel rendering over several GPUs (one process per GPU).

Camera samples are independent, so the frame shards without any exchange
inside the path tracer: rank r of N renders the samples
    sample_offset = (step * N + r) * spp_per_step, ..., + spp_per_step - 1
of every pixel into its own RGBW accumulation buffer, and one all-reduce (sum)
per step combines the ranks' buffers (NCCL over NVLink on GPUs; gloo on CPU in
the tests).  The scene is replicated per GPU.  Timing is the maximum over ranks.
Multi-scene batches shard by scene instead (rank r takes scenes r, r + N, ...),
with no exchange at all.
"""
import datetime
import os


def rank_world():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def sample_offset(step, rank, world, spp_per_step=1):
    """First sample index of this rank's share of step `step`."""
    return (step * world + rank) * spp_per_step


def shard(items, rank, world):
    """This rank's share of independent items (scenes of a batch): every N-th."""
    return list(items)[rank::world]


def init(backend, timeout_s=120.0, device=None):
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def combine(acc, dist=None):
    """Sum the ranks' RGBW accumulation buffers in place (every rank gets the total)."""
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(acc)
    return acc


def max_over_ranks(value, dist=None, device=None):
    """Maximum of a per-rank scalar (e.g. elapsed milliseconds)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
