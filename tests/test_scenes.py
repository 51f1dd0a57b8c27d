"""Seeded synthetic scene generator."""

import numpy as np

from fbme_b200 import scenes


def test_c2_scene_shapes_and_snr():
    s = scenes.config_scene("c2", 3)
    assert s.y.shape == (128, 128) and s.y.dtype == np.complex64
    assert s.x.shape == (256, 256) and np.count_nonzero(s.x) == 200
    clean = np.fft.fft2(s.x)[:128, :128]
    snr = 10 * np.log10(np.mean(np.abs(clean) ** 2) / s.noise_variance)
    assert abs(snr - 15.0) < 1e-9


def test_determinism_and_uneven_batch():
    a, b = scenes.config_scene("c1", 7), scenes.config_scene("c1", 7)
    assert np.array_equal(a.y, b.y)
    batch = scenes.uneven_batch(0, 16)
    assert len(batch) == 16
    for s in batch:
        n1, n2 = s.grid
        m1, m2 = s.y.shape
        assert (n1, n2) in scenes.UNEVEN_GRIDS
        assert 0.29 * n1 <= m1 <= 0.71 * n1 + 1 and 0.29 * n2 <= m2 <= 0.71 * n2 + 1


def test_cluster_scene():
    s = scenes.config_scene("c3", 0)
    assert s.y.shape == (256, 192) and s.grid == (512, 512)
    assert 500 < np.count_nonzero(s.x) <= 800
