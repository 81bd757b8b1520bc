import numpy as np

from gpumatting_b200.synth import batch_sizes, make_problem


def test_generator_is_deterministic_and_follows_recipe():
    a = make_problem(96, 64, 3)
    b = make_problem(96, 64, 3)
    assert np.array_equal(a.image, b.image) and np.array_equal(a.scribbles, b.scribbles)
    assert a.image.dtype == np.uint8 and a.image.shape == (64, 96, 3)
    assert set(np.unique(a.scribbles)) <= {0, 128, 255}
    frac = (a.scribbles != 128).mean()
    assert 0.05 < frac < 0.2  # ~10%; small images overshoot a little
    assert np.all(a.alpha_gt[a.scribbles == 255] > 0.98) and np.all(a.alpha_gt[a.scribbles == 0] < 0.02)
    assert np.array_equal(a.gamma != 0, a.scribbles != 128) and set(np.unique(a.gamma)) <= {0.0, 100.0}
    assert a.eps == 1e-5
    c = make_problem(96, 64, 4)
    assert not np.array_equal(a.image, c.image)


def test_batch_sizes():
    s = batch_sizes(64, seed=0)
    assert len(s) == 64 and all(256 <= w <= 1024 and 256 <= h <= 1024 for w, h in s)
    assert s == batch_sizes(64, seed=0)
