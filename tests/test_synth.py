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


def test_accuracy_fixture_matches_the_generator():
    """tests/golden/accuracy_1080p.npz holds FP64 samples of the 1920x1080
    problem; its checksum pins the generated inputs it was solved for."""
    import os
    import sys

    import numpy as np

    from gpumatting_b200.synth import make_problem

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    from make_accuracy_golden import problem_checksum

    g = np.load(os.path.join(here, "accuracy_1080p.npz"))
    p = make_problem(int(g["W"]), int(g["H"]), int(g["seed"]))
    assert np.array_equal(problem_checksum(p), g["checksum"])
    assert g["alpha64"].shape == (int(g["H"]) // int(g["stride"]), int(g["W"]) // int(g["stride"]))
    assert float(g["rel64"]) <= 1e-12
    # FP64 CG stopped at 1e-6 is ~0.3 max-abs from the FP64 solution
    assert 0.2 <= float(np.abs(g["alpha6"] - g["alpha64"]).max()) <= float(g["err6"]) <= 0.4
