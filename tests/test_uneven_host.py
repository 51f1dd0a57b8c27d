"""Host side of uneven batches and the tile-width autotuner (no GPU).

The native plan sizing (fbme_plan_workspace_bytes_ex) runs the same
grouping and validation as plan creation without touching a device, so the
Python mirror of the tile-width rule, the per-bucket workspace layout and
the error codes are checked here; the JSON cache of the autotuner runs with
an injected timer.
"""

import ctypes
import json
from math import prod

import pytest

from fbme_b200 import _native as nat
from fbme_b200.autotune import TileCache, cache_key, candidates, tune_shape, tune_shapes
from fbme_b200.config import fbme_profile_config
from fbme_b200.engine import resolve_native_config

SHAPES = [((64, 64), (32, 32)), ((128, 64), (48, 40)), ((96, 128), (40, 64)),
          ((384, 256), (180, 100)), ((1024, 512), (300, 500))]


def _sizes(shapes, params=None, cfg=None):
    lib = nat.lib()
    cfg = cfg or fbme_profile_config("stable")
    # the tensor-core stages, whose tile widths these tests probe
    c = resolve_native_config(cfg, shapes[0][0], shapes[0][1], uneven=True)
    arr = (nat.FbmeShape * len(shapes))(*[nat.FbmeShape(g[0], g[1], s[0], s[1]) for g, s in shapes])
    if params is None:
        return lib.fbme_plan_workspace_bytes_ex(arr, len(shapes), ctypes.byref(c), None, 0)
    parr = (nat.FbmeShapeParams * len(params))(*params)
    return lib.fbme_plan_workspace_bytes_ex(arr, len(shapes), ctypes.byref(c), parr, len(params))


def _param(shape, n_tile=0, iters=0):
    (g, s) = shape
    return nat.FbmeShapeParams(nat.FbmeShape(g[0], g[1], s[0], s[1]), iters, -1.0, -1, n_tile)


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0][0]}x{s[0][1]}_{s[1][0]}x{s[1][1]}")
def test_tile_width_candidates_match_the_library_rule(shape):
    ok = candidates(*shape)
    assert ok, "the default width must always be allowed for a supported shape"
    for w in (32, 64, 96, 128, 256, 512):
        n = _sizes([shape], [_param(shape, w)])
        assert (n > 0) == (w in ok), (w, ok, nat.last_error())
    # the largest grid allows only the wider tiles (at most 64 tiles per scene)
    if shape[0] == (1024, 512):
        assert 64 not in ok and 256 in ok


def test_uneven_workspace_is_the_buckets_plus_staging():
    a, b = SHAPES[0], SHAPES[1]
    one_a, one_b = _sizes([a, a]), _sizes([b])
    mixed = _sizes([a, b, a])
    assert one_a > 0 and one_b > 0
    # per-bucket layouts plus the bucket-order copies of inputs and outputs
    assert mixed > one_a + one_b
    staging_floor = 8 * (2 * prod(a[1]) + prod(b[1])) + 17 * (2 * prod(a[0]) + prod(b[0]))
    assert mixed - one_a - one_b >= staging_floor


def test_uneven_plan_rejects_a_bad_bucket():
    # polish_size 32 > N for a 4x4 grid: the bucket check names it
    assert _sizes([SHAPES[0], ((4, 4), (2, 2))]) == 0
    assert "polish_size exceeds the grid size" in nat.last_error()
    # a tile width the shape does not allow
    assert _sizes([SHAPES[0], SHAPES[1]], [_param(SHAPES[1], 96)]) == 0
    assert "dft_n_tile" in nat.last_error()


def test_shape_params_change_only_their_shape():
    a, b = SHAPES[0], SHAPES[1]
    base = _sizes([a, b])
    # a narrower tile for `a` changes its table sizes only
    narrow = _sizes([a, b], [_param(a, 64)])
    assert narrow > 0 and narrow != base
    # params for a shape not in the plan are ignored
    assert _sizes([a, b], [_param(SHAPES[2], 64)]) == base


def test_autotuner_cache_round_trip(tmp_path):
    calls = []

    def fake_timer(grid, sample, cfg, device, batch, n_tile):
        calls.append((tuple(grid), n_tile, batch))
        return {64: 3.0, 128: 1.0, 256: 2.0}[n_tile]

    cache = TileCache(tmp_path / "tune.json")
    cfg = fbme_profile_config("stable")
    shapes = [SHAPES[0], SHAPES[1], SHAPES[0]]
    best = tune_shapes(shapes, cfg, None, cache=cache, timer=fake_timer, device_name="test-device")
    assert best == {SHAPES[0]: 128, SHAPES[1]: 128}
    data = json.loads((tmp_path / "tune.json").read_text())
    assert len(data) == 2
    key = "64x64/32x32/t3/b2/test-device"
    assert data[key]["dft_n_tile"] == 128 and set(data[key]["ms"]) == {"64", "128", "256"}
    n = len(calls)

    def failing_timer(*a):
        raise AssertionError("cached shapes are not timed again")

    again = TileCache(tmp_path / "tune.json")
    assert tune_shape(*SHAPES[0], cfg, None, 2, cache=again, timer=failing_timer,
                      device_name="test-device") == 128
    assert len(calls) == n
    assert cache_key((64, 64), (32, 32), 3, 3, "dev") == "64x64/32x32/t3/b4/dev"


def test_default_width_follows_the_tile_count():
    from fbme_b200.autotune import default_width, stage_tiles

    g, s = (256, 256), (128, 128)
    assert stage_tiles(g, s, 256) == [2, 1, 2, 4]  # forward 1, forward 2, adjoint 1, adjoint 2
    # a lone scene leaves most SMs idle: the narrowest width
    assert default_width(g, s, 1, 3, 148) == 64
    # a batch whose tiles outnumber the SMs: the widest
    assert default_width(g, s, 64, 3, 148) == 256
    # the largest grid allows no narrow tile at all
    assert default_width((1024, 512), (300, 500), 1, 3, 148) == 128
    # six-term products have one width
    assert default_width(g, s, 1, 6, 148) == 128
