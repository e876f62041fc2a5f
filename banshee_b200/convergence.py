"""Time-to-relMSE measurement of the plain and the radiance-cache tracers.

The reference image is a plain GiTracer render at high spp accumulated in
float64 (each chunk of samples is summed on the device in fp32 by the
renderer, chunks are summed in float64).  To keep it affordable it covers a
centred window of the full frame at the frame's own pixel density: the window
is rendered by a camera whose image plane is exactly that window (same eye and
axes, width scaled by Wc/W, aspect Wc/Hc), so window pixel (x, y) sees the same
image-plane square as frame pixel (x0 + x, y0 + y) with x0 = (W - Wc)/2,
y0 = (H - Hc)/2.
"""
import math

import numpy as np

from . import abi
from .metrics import relmse


def window_camera(cam, W, H, Wc, Hc):
    if (W - Wc) % 2 or (H - Hc) % 2:
        raise ValueError("the window must be centred on whole pixels: W - Wc and H - Hc even")
    c = dict(cam)
    c["fovy"] = float(np.float32(2.0 * math.atan(math.tan(cam["fovy"] * 0.5) * Wc / W)))
    c["aspect"] = Wc / Hc
    return c


def window_slice(W, H, Wc, Hc):
    """Rows/cols of the (row-flipped) frame accumulation buffer that hold the window."""
    x0, y0 = (W - Wc) // 2, (H - Hc) // 2
    return slice(H - y0 - Hc, H - y0), slice(x0, x0 + Wc)


def ground_truth(gs, Wc, Hc, spp, maxdepth, seed, chunk=256, camera=None):
    """float64 mean image (Hc, Wc, 3) of a plain render at `spp` samples per pixel."""
    import torch
    from .scene import camera_desc
    cam = camera_desc(camera) if camera is not None else None
    acc64 = torch.zeros((Hc, Wc, 4), dtype=torch.float64, device="cuda")
    acc32 = torch.zeros((Hc, Wc, 4), dtype=torch.float32, device="cuda")
    for off in range(0, spp, chunk):
        acc32.zero_()
        n = min(chunk, spp - off)
        gs.render(acc32.data_ptr(), Wc, Hc, n, seed=seed, sample_offset=off, maxdepth=maxdepth, camera=cam,
                  stats=False)
        acc64 += acc32.double()
    torch.cuda.synchronize()
    a = acc64.cpu().numpy()
    return a[..., :3] / a[..., 3:4]


def converge(render_frame, W, H, Wc, Hc, gt, max_seconds, max_frames, target=1e-3, every=1):
    """Renders frames (render_frame(acc_ptr, frame_index)) until relMSE on the
    window <= target or a budget runs out.  Time is the sum of CUDA-event times
    of the render calls.  Returns dict(curve=[(t_s, frames, relmse)], t_target)."""
    import torch
    acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    rs, cs = window_slice(W, H, Wc, Hc)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t = 0.0
    curve = []
    t_target = None
    for f in range(max_frames):
        e0.record()
        render_frame(acc.data_ptr(), f)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) * 1e-3
        if (f + 1) % every == 0 or f + 1 == max_frames:
            win = acc[rs, cs].double().cpu().numpy()
            img = win[..., :3] / np.maximum(win[..., 3:4], 1.0)
            e = relmse(img, gt)
            curve.append((t, f + 1, e))
            if e <= target and t_target is None:
                # linear interpolation in log(relMSE) between the last two points
                if len(curve) >= 2 and curve[-2][2] > target:
                    (ta, _, ea), (tb, _, eb) = curve[-2], curve[-1]
                    w = (math.log(ea) - math.log(target)) / max(math.log(ea) - math.log(eb), 1e-12)
                    t_target = ta + w * (tb - ta)
                else:
                    t_target = t
                break
        if t > max_seconds:
            break
    return {"curve": curve, "t_target": t_target, "frames": curve[-1][1] if curve else 0,
            "final_relmse": curve[-1][2] if curve else None, "seconds": t}


# ---------------------------------------------------------------- full frame
def converge_frame(render_frame, W, H, gt, gt_var, max_seconds, max_frames, target=1e-3, every=1):
    """Full-frame version of converge(): relMSE of the whole W x H image against
    the float64 reference `gt` (H, W, 3, a device tensor, in the accumulation
    buffer's row order) with the reference's own variance `gt_var` subtracted
    (groundtruth.relmse_vs).  The time is the CUDA-event time of the render
    calls only; the error evaluation runs outside it."""
    import torch
    from .groundtruth import relmse_vs
    acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t = 0.0
    curve = []
    t_target = None
    for f in range(max_frames):
        e0.record()
        render_frame(acc.data_ptr(), f)
        e1.record()
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) * 1e-3
        if (f + 1) % every == 0 or f + 1 == max_frames:
            img = acc[..., :3].double() / acc[..., 3:4].double().clamp(min=1.0)
            _, e = relmse_vs(img, gt, gt_var)
            curve.append((t, f + 1, e))
            if e <= target and t_target is None:
                if len(curve) >= 2 and curve[-2][2] > target:
                    (ta, _, ea), (tb, _, eb) = curve[-2], curve[-1]
                    w = (math.log(ea) - math.log(target)) / max(math.log(ea) - math.log(eb), 1e-12)
                    t_target = ta + w * (tb - ta)
                else:
                    t_target = t
                break
        if t > max_seconds:
            break
    return {"curve": curve, "t_target": t_target, "frames": curve[-1][1] if curve else 0,
            "final_relmse": curve[-1][2] if curve else None, "seconds": t}


def bias_floor(render_frame, W, H, gt, gt_var, frames, first_frame=0):
    """Error floor of a (possibly biased) renderer: renders `frames` frames
    (render_frame(acc_ptr, frame_index), frame indices from first_frame) into
    two buffers by frame parity and splits the relMSE of their combined image
    against the reference into its noise (the halves' difference estimates the
    image's own variance) and the rest, the squared bias:
        relmse = bias^2 + Var(image) + Var(reference).
    Returns dict(relmse, image_noise, reference_noise, bias_floor)."""
    import torch
    from .metrics import RELMSE_EPS
    halves = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    for f in range(frames):
        render_frame(halves[f & 1].data_ptr(), first_frame + f)
    torch.cuda.synchronize()
    a, b = (x.double() for x in halves)
    ma = a[..., :3] / a[..., 3:4].clamp(min=1.0)
    mb = b[..., :3] / b[..., 3:4].clamp(min=1.0)
    tot = a + b
    m = tot[..., :3] / tot[..., 3:4].clamp(min=1.0)
    w = 1.0 / (gt * gt + RELMSE_EPS)
    raw = float(((m - gt) ** 2 * w).mean())
    noise = float(((ma - mb) ** 2 / 4.0 * w).mean())
    ref_noise = float((gt_var * w).mean())
    return {"frames": frames, "relmse": raw, "image_noise": noise, "reference_noise": ref_noise,
            "bias_floor": raw - noise - ref_noise}
