"""Float64 accumulation of a progressive render, with checkpoint and resume.

The radiance cache is measured against a plain GiTracer render at high spp
accumulated in float64.  At 1080p and 65,536 spp that is 1.36e11 camera
samples, minutes of GPU time, so the accumulation is resumable:

* the renderer adds `chunk` samples per pixel into an fp32 RGBW buffer (its own
  sum, as FileImagePlane::WriteSample adds, imageplane/fileimageplane.cpp:29-34);
  each chunk is then added into one of two float64 halves (even and odd
  chunks), so the float32 sums never span more than one chunk;
* every `every` chunks (and at the end) the halves, the samples done and a key
  naming what is accumulated (scene, camera, size, depth, seed) are written to
  a checkpoint file, atomically (temporary file + rename); a later run with the
  same key resumes from it, a different key starts over;
* the two halves give the estimate's own variance: with equal halves A and B,
  the variance of the combined mean is about (mean_A - mean_B)^2 / 4 per pixel
  and channel, which the relMSE of an image against this reference can subtract.

Works on any torch device (the GPU in the benchmark, the CPU in the tests).
"""
import json
import os

import numpy as np

from .metrics import RELMSE_EPS


class Fp64Accumulator:
    def __init__(self, height, width, key, device="cuda"):
        import torch
        self.shape = (height, width)
        self.key = json.dumps(key, sort_keys=True)
        self.device = device
        self.half = [torch.zeros((height, width, 4), dtype=torch.float64, device=device) for _ in range(2)]
        self.chunks = 0          # chunks added
        self.spp = 0             # samples per pixel added

    def add(self, acc32, spp):
        """Adds one fp32 RGBW chunk of `spp` samples per pixel."""
        self.half[self.chunks & 1] += acc32.double()
        self.chunks += 1
        self.spp += int(spp)

    def save(self, path):
        tmp = path + ".tmp"
        with open(tmp, "wb") as f:
            np.savez(f, a=self.half[0].cpu().numpy(), b=self.half[1].cpu().numpy(),
                     meta=np.frombuffer(json.dumps({"key": self.key, "chunks": self.chunks,
                                                    "spp": self.spp}).encode(), dtype=np.uint8))
        os.replace(tmp, path)

    def load(self, path):
        """Resumes from `path` if it holds the same key; returns True if it did."""
        import torch
        if not path or not os.path.exists(path):
            return False
        with np.load(path) as z:
            meta = json.loads(bytes(z["meta"]).decode())
            if meta["key"] != self.key or z["a"].shape[:2] != self.shape:
                return False
            self.half[0] = torch.from_numpy(z["a"]).to(self.device)
            self.half[1] = torch.from_numpy(z["b"]).to(self.device)
        self.chunks, self.spp = int(meta["chunks"]), int(meta["spp"])
        return True

    def _means(self):
        a, b = self.half
        ma = a[..., :3] / a[..., 3:4].clamp(min=1.0)
        mb = b[..., :3] / b[..., 3:4].clamp(min=1.0)
        tot = a + b
        return tot[..., :3] / tot[..., 3:4].clamp(min=1.0), ma, mb

    def mean(self):
        """float64 mean image (H, W, 3) on the accumulator's device."""
        return self._means()[0]

    def mean_variance(self):
        """Per-pixel, per-channel variance of mean() estimated from the halves."""
        m, ma, mb = self._means()
        return (ma - mb) ** 2 / 4.0


def accumulate(render_chunk, height, width, spp, key, chunk=256, path=None, every=16, device="cuda",
               on_chunk=None):
    """Accumulates `spp` samples per pixel in chunks: render_chunk(acc32, sample_offset, n)
    adds n samples per pixel, starting at sample index sample_offset, into the
    zeroed fp32 RGBW tensor acc32.  Resumes from / checkpoints to `path` (None:
    no checkpoint).  Returns the accumulator."""
    import torch
    acc = Fp64Accumulator(height, width, key, device=device)
    acc.load(path)
    acc32 = torch.zeros((height, width, 4), dtype=torch.float32, device=device)
    since = 0
    while acc.spp < spp:
        n = min(chunk, spp - acc.spp)
        acc32.zero_()
        render_chunk(acc32, acc.spp, n)
        acc.add(acc32, n)
        since += 1
        if on_chunk:
            on_chunk(acc)
        if path and since >= every:
            acc.save(path)
            since = 0
    if path and since:
        acc.save(path)
    return acc


def relmse_vs(img, ref, ref_var=None, eps=RELMSE_EPS):
    """relMSE of `img` (H, W, 3) against `ref`, mean over pixels and channels of
    (x - ref)^2 / (ref^2 + eps), on the tensors' device.  With `ref_var` (the
    reference's own per-pixel variance, Fp64Accumulator.mean_variance) also the
    same value with the reference's noise subtracted: E[(x - ref)^2] = the
    squared error against the true image + Var(ref).  Returns (raw, corrected)."""
    w = 1.0 / (ref * ref + eps)
    raw = float(((img.double() - ref) ** 2 * w).mean())
    if ref_var is None:
        return raw, raw
    return raw, raw - float((ref_var * w).mean())
