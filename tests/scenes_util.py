"""Seeded synthetic scenes for the tests (fbme_b200.scenes)."""

import numpy as np


def c1_scene(seed: int):
    """64 x 64 grid, 32 x 32 prefix, 40 CN(0, 1) points, 20 dB: (y, grid)."""
    from fbme_b200 import scenes

    sc = scenes.config_scene("c1", seed)
    return np.ascontiguousarray(sc.y.astype(np.complex64)), tuple(sc.grid)
