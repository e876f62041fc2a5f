"""Checkpointed float64 accumulation of the reference image (groundtruth.py),
on CPU with the oracle as the renderer: a run interrupted after a checkpoint
and resumed gives the same float64 sums, bit for bit, as an uninterrupted run;
a checkpoint of something else (another key) is not resumed; the result
equals one render of all the samples up to float32 summation order."""
import numpy as np


def _renderer(o, log):
    def render_chunk(acc32, offset, n):
        log.append((offset, n))
        o.render(spp=n, seed=5, maxdepth=5, sample_offset=offset, accum=acc32.numpy(), nthreads=1)
    return render_chunk


def test_resume_from_checkpoint_equals_uninterrupted(tmp_path, oracle_built):
    from banshee_b200 import groundtruth as GT
    from banshee_b200 import scenes
    sc = scenes.cornell(16, 16)
    o = oracle_built.Oracle(sc)
    key = {"scene": sc.name, "w": 16, "h": 16, "depth": 5, "seed": 5}
    path = str(tmp_path / "gt.npz")

    log_full = []
    full = GT.accumulate(_renderer(o, log_full), 16, 16, 8, key, chunk=2, device="cpu")
    assert log_full == [(0, 2), (2, 2), (4, 2), (6, 2)] and full.spp == 8

    log_a = []
    part = GT.accumulate(_renderer(o, log_a), 16, 16, 4, key, chunk=2, path=path, every=1, device="cpu")
    assert part.spp == 4 and log_a == [(0, 2), (2, 2)]
    log_b = []
    resumed = GT.accumulate(_renderer(o, log_b), 16, 16, 8, key, chunk=2, path=path, every=1, device="cpu")
    assert log_b == [(4, 2), (6, 2)]                         # only the missing samples are rendered
    for h in range(2):
        assert (resumed.half[h].numpy() == full.half[h].numpy()).all()

    # another key does not resume
    log_c = []
    other = GT.accumulate(_renderer(o, log_c), 16, 16, 2, dict(key, seed=6), chunk=2, path=path, device="cpu")
    assert log_c == [(0, 2)] and other.spp == 2

    one = o.render(spp=8, seed=5, maxdepth=5, nthreads=1)
    m = full.mean().numpy()
    ref = one[..., :3] / one[..., 3:4]
    np.testing.assert_allclose(m, ref, rtol=1e-5, atol=1e-6)
    assert (full.mean_variance().numpy() >= 0).all()


def test_relmse_with_reference_noise_subtracted():
    import torch
    from banshee_b200 import groundtruth as GT
    rng = np.random.default_rng(1)
    truth = torch.from_numpy(rng.random((32, 32, 3)) + 0.1)
    ref_var = torch.full_like(truth, 1e-4)
    raw, corr = GT.relmse_vs(truth, truth)
    assert raw == 0.0 and corr == 0.0
    raw, corr = GT.relmse_vs(truth + 0.01, truth, ref_var)
    assert corr < raw and abs(raw - corr - float((ref_var / (truth * truth + 0.01)).mean())) < 1e-12
