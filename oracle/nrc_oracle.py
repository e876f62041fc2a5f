"""CPU oracle of the neural radiance cache -- TEST INFRASTRUCTURE ONLY.

The cache has no counterpart in the reference (Banshee has no learned part).
This restates, in float64 numpy, the published algorithms the GPU kernels
implement (banshee_b200/csrc/cache.cu):
  * multiresolution hash-grid encoding (Mueller et al. 2022, "Instant Neural
    Graphics Primitives"): per level l, resolution N_l = floor(N_min * b^l),
    trilinear interpolation of 2 features at the 8 cell corners, dense index
    when (N_l + 1)^3 <= T, else (x * 1 ^ y * 2654435761 ^ z * 805459861) mod T;
  * one-blob encoding (Mueller et al. 2019, "Neural Importance Sampling") of
    spherical coordinates with 16 Gaussian bins (sigma = 1/16);
  * a bias-free ReLU MLP 128-64-64-64-64-64-16 with the relative L2 loss of
    neural radiance caching (Mueller et al. 2021);
and emulates bf16 rounding (round to nearest even) at the points where the GPU
rounds: encoded inputs, hidden activations, weights, and back-propagated
layer gradients.  Accumulation is float64.
"""
import numpy as np

LEVELS, FEAT, IN, H, OUT = 16, 2, 128, 64, 16
W_SHAPES = [(64, 128), (64, 64), (64, 64), (64, 64), (64, 64), (16, 64)]
W_OFFS = np.cumsum([0] + [a * b for a, b in W_SHAPES])
NPARAMS = int(W_OFFS[-1])


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


def resolutions(base, finest):
    b = np.exp((np.log(finest) - np.log(base)) / (LEVELS - 1))
    return [int(np.floor(base * b ** l)) for l in range(LEVELS)]


def unpack(w):
    return [w[W_OFFS[i]:W_OFFS[i + 1]].reshape(W_SHAPES[i]) for i in range(6)]


def _grid_corners(u, res, log2_t):
    """Per level: list of (index array, weight array) for the 8 corners."""
    T = 1 << log2_t
    N = float(res)
    x = u * np.float32(N)
    x0 = np.minimum(np.floor(x), N - 1)
    f = x - x0
    x0 = x0.astype(np.int64)
    out = []
    for cidx in range(8):
        d = np.array([cidx & 1, (cidx >> 1) & 1, (cidx >> 2) & 1])
        w = np.prod(np.where(d[None, :] == 1, f, 1 - f), axis=1)
        c = x0 + d[None, :]
        n1 = res + 1
        if n1 ** 3 <= T:
            idx = c[:, 0] + n1 * (c[:, 1] + n1 * c[:, 2])
        else:
            idx = ((c[:, 0].astype(np.uint32) * np.uint32(1)) ^ (c[:, 1].astype(np.uint32) * np.uint32(2654435761))
                   ^ (c[:, 2].astype(np.uint32) * np.uint32(805459861))) & np.uint32(T - 1)
        out.append((idx.astype(np.int64), w))
    return out


def normalize_pos(p, bmin, bscale):
    return np.clip((p.astype(np.float32) - bmin) * bscale, 0.0, 1.0).astype(np.float32)


def one_blob(v):
    centers = (np.arange(16) + 0.5) / 16.0
    d = v[:, None] - centers[None, :]
    return np.exp(-d * d * 128.0)


def sph(w):
    th = np.arccos(np.clip(w[:, 2], -1, 1)) / np.pi
    ph = np.arctan2(w[:, 1], w[:, 0]) / (2 * np.pi) + 0.5
    return th, ph


def encode(feat, grid, res, log2_t, bmin, bscale):
    """feat (n, 16) -> bf16-rounded encoded inputs (n, 128) and the grid corner data."""
    n = feat.shape[0]
    X = np.zeros((n, IN))
    u = normalize_pos(feat[:, 0:3], bmin, bscale)
    T = 1 << log2_t
    g = grid.reshape(LEVELS, T, FEAT).astype(np.float64)
    corners = []
    for l in range(LEVELS):
        cs = _grid_corners(u, res[l], log2_t)
        corners.append(cs)
        acc = np.zeros((n, FEAT))
        for idx, w in cs:
            acc += w[:, None] * g[l, idx]
        X[:, 2 * l:2 * l + 2] = acc
    th, ph = sph(feat[:, 3:6])
    X[:, 32:48] = one_blob(th)
    X[:, 48:64] = one_blob(ph)
    th, ph = sph(feat[:, 6:9])
    X[:, 64:80] = one_blob(th)
    X[:, 80:96] = one_blob(ph)
    X[:, 96:100] = feat[:, 9:13]
    X[:, 100] = 1.0
    return bf16(X), corners


def forward(X, w):
    Ws = [bf16(W) for W in unpack(np.asarray(w, dtype=np.float64))]
    hs = [X]
    a = X
    for W in Ws[:5]:
        a = bf16(np.maximum(a @ W.T, 0.0))
        hs.append(a)
    out = a @ Ws[5].T
    return out, hs, Ws


def loss_and_grads(feat, target, w, grid, res, log2_t, bmin, bscale):
    """Relative L2 loss and float64 gradients of the MLP weights and the grid."""
    n = feat.shape[0]
    X, corners = encode(feat, grid, res, log2_t, bmin, bscale)
    out, hs, Ws = forward(X, w)
    p = out[:, :3]
    y = target[:, :3]
    den = p * p + 0.01
    loss = np.sum((p - y) ** 2 / den) / (3 * n)
    g = np.zeros((n, OUT))
    g[:, :3] = 2 * (p - y) / den / (3 * n)
    dz = bf16(g)
    dW = [None] * 6
    dW[5] = dz.T @ hs[5]
    dh = dz @ Ws[5]
    for l in range(4, -1, -1):
        dz = bf16(np.where(hs[l + 1] > 0, dh, 0.0))
        dW[l] = dz.T @ hs[l]
        dh = dz @ Ws[l]
    dX = dh[:, :32]
    T = 1 << log2_t
    dgrid = np.zeros((LEVELS, T, FEAT))
    for l in range(LEVELS):
        for idx, wgt in corners[l]:
            np.add.at(dgrid[l], idx, wgt[:, None] * dX[:, 2 * l:2 * l + 2])
    return loss, np.concatenate([d.reshape(-1) for d in dW]), dgrid.reshape(-1), out
