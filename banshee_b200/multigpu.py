"""Data-parallel rendering over several GPUs (one process per GPU).

Camera samples are independent, so the frame shards without any exchange
inside the path tracer: rank r of N renders the samples
    sample_offset = (step * N + r) * spp_per_step, ..., + spp_per_step - 1
of every pixel into a zeroed per-step RGBW buffer; one all-reduce (sum) of
that buffer per step combines the ranks' samples of the step, and the sum is
added once into the running total (``StepExchange``; NCCL over NVLink on GPUs,
gloo on CPU in the tests).  Every sample is therefore added exactly once, as
FileImagePlane::WriteSample adds it (imageplane/fileimageplane.cpp:29-34).  The scene is replicated per GPU.  Timing is the maximum over ranks.
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


def _distributed(dist):
    return dist is not None and dist.is_initialized() and dist.get_world_size() > 1


def combine(acc, dist=None):
    """Sum the ranks' RGBW buffers in place (every rank gets the total).  Use it
    once on buffers that each hold only their own rank's samples; for a running
    total that is combined every step use StepExchange."""
    if _distributed(dist):
        dist.all_reduce(acc)
    return acc


class StepExchange:
    """Per-step exchange of a progressive render over N ranks.

    ``target`` is the buffer a step renders into.  With one rank it is the
    running total itself (no exchange).  With N ranks it is a per-step buffer:
    ``end_step()`` all-reduces it (each rank's samples of this step), adds the
    sum into ``total`` and clears it for the next step, so a sample reaches the
    total once however many steps follow.  Every rank holds the same total."""

    def __init__(self, total, dist=None):
        self.total = total
        self.dist = dist
        self.exchange = _distributed(dist)
        self.target = total.new_zeros(total.shape) if self.exchange else total

    def end_step(self):
        if self.exchange:
            self.dist.all_reduce(self.target)
            self.total.add_(self.target)
            self.target.zero_()
        return self.total


def max_over_ranks(value, dist=None, device=None):
    """Maximum of a per-rank scalar (e.g. elapsed milliseconds)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
