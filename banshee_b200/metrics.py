"""Image metrics used by the tests and the benchmark."""
import numpy as np

RELMSE_EPS = 0.01


def mean_image(accum):
    """RGBW accumulation buffer -> per-pixel mean RGB (float64)."""
    a = np.asarray(accum, dtype=np.float64)
    w = np.maximum(a[..., 3:4], 1.0)
    return a[..., :3] / w


def relmse(img, ref, eps=RELMSE_EPS):
    """mean over pixels and channels of (x - ref)^2 / (ref^2 + eps)."""
    x = np.asarray(img, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + eps)))
