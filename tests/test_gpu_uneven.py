"""Uneven batches and tuned tile widths on the B200.

An uneven plan groups its scenes into one bucket per shape; its UAMP steps
run as launches merged over the buckets and each bucket's polish as its own
equal-shape batch.  Scenes are independent, so every scene's result must
equal, bit for bit, the result of an equal-shape plan holding that shape's
scenes in the same order.  Odd shapes (non-square grids,
prefix lengths that are not multiples of the tile sizes) are checked
against the oracle at the parity bar: identical support, x within 1e-4
relative L2, posterior variance within 1e-3 on the support.  The tile
width changes only the grouping of the per-tile partial sums, so plans
with 64-, 128- and 256-column tiles agree to rounding and all meet the bar.
"""

import numpy as np
import pytest

from gpu_util import PV_TOL, X_TOL, need_gpu, rel_l2

torch = pytest.importorskip("torch")

A = ((64, 64), (32, 32))
B = ((128, 64), (48, 40))
C = ((96, 128), (24, 64))
ORDER = [A, B, A, C, B, A]


def _scenes(shapes, seed0=500):
    from fbme_b200 import scenes

    out = []
    for i, (g, s) in enumerate(shapes):
        k = max(8, int(0.02 * g[0] * g[1]))
        out.append(scenes.point_scene(g, s, k, 15.0, seed0 + i, "cn"))
    return out


def _cfg(profile="stable"):
    """The profile with the tensor-core stages, which uneven plans run, so
    that the equal-shape references run the same arithmetic."""
    from fbme_b200.config import fbme_profile_config

    cfg = fbme_profile_config(profile)
    cfg.dft_terms = 3
    return cfg


FIELDS_PIX = ("x", "posterior_variance", "precision", "support_mask")
FIELDS_SCENE = ("noise_variance", "effective_dof", "negative_log_evidence", "evidence_trace",
                "support_exchanges_accepted", "fixed_budget_gamma_residual", "fixed_budget_noise_residual",
                "fixed_budget_objective_decrease", "fixed_budget_monotone", "support_score_threshold",
                "active_indices", "status")


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
def test_uneven_plan_equals_per_shape_plans(profile):
    need_gpu()
    from fbme_b200.engine import FBMEEngine, uamp_iteration_limit
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    cfg = _cfg(profile)
    sc = _scenes(ORDER)
    eng = UnevenEngine(ORDER, cfg, dev)
    y = eng.pack([torch.from_numpy(s.y).to(dev) for s in sc])
    eng.run(y)
    torch.cuda.synchronize()
    # buckets in order of first appearance, with the shape's own T_u
    bk = eng.buckets()
    assert [(b["grid"], b["sample"], b["scenes"]) for b in bk] == [(A[0], A[1], 3), (B[0], B[1], 2),
                                                                 (C[0], C[1], 1)]
    for b in bk:
        assert b["uamp_iterations"] == uamp_iteration_limit(cfg, b["grid"][0] * b["grid"][1],
                                                             b["sample"][0] * b["sample"][1])
    assert len({b["uamp_iterations"] for b in bk}) > 1  # the scenes stop at different sweeps
    for shape in (A, B, C):
        idx = [i for i, s in enumerate(ORDER) if s == shape]
        ref = FBMEEngine(len(idx), shape[0], shape[1], cfg, dev)
        ys = torch.stack([torch.from_numpy(sc[i].y).to(dev) for i in idx]).reshape(len(idx), -1)
        ref.run(ys.contiguous())
        torch.cuda.synchronize()
        n = shape[0][0] * shape[0][1]
        for j, i in enumerate(idx):
            p0 = eng.pix_off[i]
            for f in FIELDS_PIX:
                assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][j]), (f, i)
            for f in FIELDS_SCENE:
                assert torch.equal(eng.out[f][i], ref.out[f][j]), (f, i)
        ref.close()
    assert int(eng.out["status"].abs().sum()) == 0
    eng.close()


@pytest.mark.gpu
def test_uneven_graph_replay_and_results():
    need_gpu()
    from fbme_b200.uneven import UnevenEngine, make_uneven_plan

    dev = torch.device("cuda", 0)
    sc = _scenes(ORDER, 900)
    ys = [torch.from_numpy(s.y).to(dev) for s in sc]
    plan = make_uneven_plan(ys, [s[0] for s in ORDER], warmup=1)
    res = plan.replay(ys, synchronize=True)
    assert len(res) == len(ORDER)
    for r, (g, _) in zip(res, ORDER):
        assert tuple(r.x.shape) == g and r.x.dtype == torch.complex64
    eager = UnevenEngine(ORDER, plan.config, dev)
    eager.run(eager.pack(ys))
    torch.cuda.synchronize()
    for f in FIELDS_PIX + FIELDS_SCENE:
        assert torch.equal(plan.engine.out[f], eager.out[f]), f
    # new data through the packed entry point, then the first data again
    other = [torch.from_numpy(s.y).to(dev) for s in _scenes(ORDER, 950)]
    x0 = res[3].x.clone()
    plan.replay(torch.cat([o.reshape(-1) for o in other]), synchronize=True)
    assert not torch.equal(plan.result[3].x, x0)
    plan.replay(ys, synchronize=True)
    assert torch.equal(plan.result[3].x, x0)
    eager.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [B, C], ids=["128x64_48x40", "96x128_24x64"])
def test_uneven_scene_matches_oracle(shape):
    need_gpu()
    from fbme_b200.uneven import UnevenEngine
    from oracle import fbme_oracle as O

    dev = torch.device("cuda", 0)
    order = [A, shape, A]
    sc = _scenes(order, 1300)
    eng = UnevenEngine(order, _cfg(), dev)
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    res = eng.results()
    for i in (0, 1):
        g = order[i][0]
        ref = O.fbme_solve(sc[i].y[None], g, "stable")
        x = res[i].x.cpu().numpy().reshape(-1)
        xr = ref["x"].reshape(-1)
        assert set(np.flatnonzero(x)) == set(np.flatnonzero(xr))
        assert rel_l2(x, xr) < X_TOL
        pv = res[i].posterior_variance.cpu().numpy().reshape(-1)
        pvr = ref["posterior_variance"].reshape(-1)
        sup = xr != 0
        assert np.max(np.abs(pv[sup] - pvr[sup]) / pvr[sup]) < PV_TOL
        assert res[i].iterations == int(ref["iterations"])
    eng.close()


@pytest.mark.gpu
def test_tile_widths_agree_and_meet_the_bar():
    need_gpu()
    from fbme_b200.autotune import candidates
    from fbme_b200.engine import FBMEEngine
    from oracle import fbme_oracle as O

    dev = torch.device("cuda", 0)
    shape = B
    sc = _scenes([shape] * 3, 1700)
    y_np = np.stack([s.y for s in sc])
    y = torch.from_numpy(y_np).to(dev).reshape(3, -1).contiguous()
    xs = {}
    for w in candidates(*shape):
        e = FBMEEngine(3, shape[0], shape[1], _cfg(), dev, n_tile=w)
        e.run(y)
        torch.cuda.synchronize()
        xs[w] = e.out["x"].cpu().numpy()
        assert int(e.out["status"].abs().sum()) == 0
        e.close()
    assert set(xs) == {64, 128, 256}
    ref = O.fbme_solve(y_np, shape[0], "stable")["x"].reshape(3, -1)
    for w, x in xs.items():
        for i in range(3):
            assert set(np.flatnonzero(x[i])) == set(np.flatnonzero(ref[i])), w
            assert rel_l2(x[i], ref[i]) < X_TOL, w
            assert rel_l2(x[i], xs[256][i]) < 1e-5, w


@pytest.mark.gpu
def test_autotuner_times_every_width_and_caches(tmp_path):
    need_gpu()
    from fbme_b200.autotune import TileCache, candidates, tune_shape

    dev = torch.device("cuda", 0)
    cache = TileCache(tmp_path / "tune.json")
    best = tune_shape(A[0], A[1], _cfg(), dev, 8, cache=cache)
    assert best in candidates(*A)
    (entry,) = cache.entries.values()
    assert set(entry["ms"]) == {str(w) for w in candidates(*A)}
    assert all(t > 0 for t in entry["ms"].values())
    assert entry["ms"][str(best)] == min(entry["ms"].values())


D = ((64, 64), (31, 33))
E = ((128, 64), (45, 37))


@pytest.mark.gpu
def test_odd_sample_counts_in_an_uneven_plan():
    """Odd M puts scenes at 8-byte (not 16-byte) offsets of the packed
    samples; each bucket's copy starts aligned, and scene rows with odd
    strides take the scalar path."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    order = [D, E, D, A]
    sc = _scenes(order, 2100)
    eng = UnevenEngine(order, _cfg(), dev)
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    for shape in (D, E):
        idx = [i for i, s in enumerate(order) if s == shape]
        ref = FBMEEngine(len(idx), shape[0], shape[1], _cfg(), dev)
        ref.run(torch.stack([torch.from_numpy(sc[i].y).to(dev) for i in idx]).reshape(len(idx), -1).contiguous())
        torch.cuda.synchronize()
        n = shape[0][0] * shape[0][1]
        for j, i in enumerate(idx):
            assert torch.equal(eng.out["x"][eng.pix_off[i]:eng.pix_off[i] + n], ref.out["x"][j])
            assert torch.equal(eng.out["negative_log_evidence"][i], ref.out["negative_log_evidence"][j])
        ref.close()
    eng.close()


@pytest.mark.gpu
def test_samples_at_an_8_byte_offset():
    """A caller's complex64 pointer need only be 8-byte aligned: stages
    that read y fall back to 8-byte accesses and give the same result."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine

    dev = torch.device("cuda", 0)
    sc = _scenes([A, A], 2200)
    y = torch.stack([torch.from_numpy(s.y).to(dev) for s in sc]).reshape(2, -1).contiguous()
    buf = torch.zeros(y.numel() + 1, dtype=torch.complex64, device=dev)
    buf[1:].copy_(y.reshape(-1))
    view = buf[1:].view(2, -1)
    assert view.data_ptr() % 16 == 8
    eng = FBMEEngine(2, A[0], A[1], _cfg(), dev)
    eng.run(y)
    torch.cuda.synchronize()
    x0 = eng.out["x"].clone()
    eng.run(view)
    torch.cuda.synchronize()
    assert torch.equal(eng.out["x"], x0)
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [((32, 320), (16, 100)), ((48, 63), (20, 30))],
                         ids=["32x320_16x100", "48x63_20x30"])
def test_exchange_tile_classes_match_oracle(shape):
    """The residual-exchange scoring has one tile class per N2 range; rows
    wider than 256 (the 16-row class) and odd N2 (8-byte row staging) meet
    the parity bar against the oracle, with the Stable profile's exchange."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from oracle import fbme_oracle as O

    dev = torch.device("cuda", 0)
    g = shape[0]
    sc = _scenes([shape] * 3, 2500)
    y_np = np.stack([s.y for s in sc])
    eng = FBMEEngine(3, shape[0], shape[1], _cfg(), dev)
    eng.run(torch.from_numpy(y_np).to(dev).reshape(3, -1).contiguous())
    torch.cuda.synchronize()
    assert int(eng.out["status"].abs().sum()) == 0
    x = eng.out["x"].cpu().numpy().reshape(3, -1)
    pv = eng.out["posterior_variance"].cpu().numpy().reshape(3, -1)
    ref = O.fbme_solve(y_np, g, "stable")
    xr = ref["x"].reshape(3, -1)
    pvr = ref["posterior_variance"].reshape(3, -1)
    for i in range(3):
        assert set(np.flatnonzero(x[i])) == set(np.flatnonzero(xr[i])), i
        assert rel_l2(x[i], xr[i]) < X_TOL, i
        sup = xr[i] != 0
        assert np.max(np.abs(pv[i][sup] - pvr[i][sup]) / pvr[i][sup]) < PV_TOL, i
    np.testing.assert_array_equal(eng.out["support_exchanges_accepted"].cpu().numpy(),
                                  np.asarray(ref["support_exchanges_accepted"]).reshape(-1))
    eng.close()


@pytest.mark.gpu
def test_more_buckets_than_one_merged_launch_holds():
    """70 distinct shapes: the merged UAMP launches take at most 64 buckets
    each, so every step splits into two launches; every scene still equals
    its own single-scene plan bit for bit, and the buckets stop at
    different sweeps."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(31)
    shapes = []
    while len(shapes) < 70:
        g = (int(rng.choice([32, 40, 48, 64])), int(rng.choice([32, 48, 56, 64, 80])))
        s = (int(rng.integers(8, g[0] // 2 + 1)), int(rng.integers(8, g[1] // 2 + 1)))
        if (g, s) not in shapes:
            shapes.append((g, s))
    sc = _scenes(shapes, 2100)
    cfg = _cfg()
    eng = UnevenEngine(shapes, cfg, dev)
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert len(eng.buckets()) == 70
    assert len({b["uamp_iterations"] for b in eng.buckets()}) > 1
    assert int(eng.out["status"].abs().sum()) == 0
    for i in range(0, 70, 3):
        g, s = shapes[i]
        ref = FBMEEngine(1, g, s, cfg, dev, n_tile=eng.tile_widths[(g, s)])
        ref.run(torch.from_numpy(sc[i].y).to(dev).reshape(1, -1).contiguous())
        torch.cuda.synchronize()
        p0, n = eng.pix_off[i], g[0] * g[1]
        for f in FIELDS_PIX:
            assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][0]), (f, i)
        for f in FIELDS_SCENE:
            assert torch.equal(eng.out[f][i], ref.out[f][0]), (f, i)
        ref.close()
    eng.close()


@pytest.mark.gpu
def test_buckets_with_different_tile_widths():
    """Buckets laid out for 64-, 128- and 256-column tiles: each merged UAMP
    step splits into one launch per width, and every scene still equals the
    equal-shape plan of its width bit for bit."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    widths = {A: 64, B: 128, C: 256}
    sc = _scenes(ORDER, 2600)
    cfg = _cfg()
    eng = UnevenEngine(ORDER, cfg, dev, tile_widths=widths)
    assert {sh: eng.tile_widths[sh] for sh in widths} == widths
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert int(eng.out["status"].abs().sum()) == 0
    for shape, w in widths.items():
        idx = [i for i, s in enumerate(ORDER) if s == shape]
        ref = FBMEEngine(len(idx), shape[0], shape[1], cfg, dev, n_tile=w)
        ys = torch.stack([torch.from_numpy(sc[i].y).to(dev) for i in idx]).reshape(len(idx), -1)
        ref.run(ys.contiguous())
        torch.cuda.synchronize()
        n = shape[0][0] * shape[0][1]
        for j, i in enumerate(idx):
            p0 = eng.pix_off[i]
            for f in FIELDS_PIX:
                assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][j]), (f, i, w)
            for f in FIELDS_SCENE:
                assert torch.equal(eng.out[f][i], ref.out[f][j]), (f, i, w)
        ref.close()
    eng.close()


@pytest.mark.gpu
def test_six_term_buckets_match_per_shape_plans():
    """6-term DFT products (BF16 hi/mid/lo) in an uneven plan: the merged
    steps take the 6-term stage launches, and every scene equals the
    equal-shape 6-term plan bit for bit."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    cfg = _cfg()
    cfg.dft_terms = 6
    order = [A, C, A]
    sc = _scenes(order, 2900)
    eng = UnevenEngine(order, cfg, dev)
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert int(eng.out["status"].abs().sum()) == 0
    for shape in (A, C):
        idx = [i for i, s in enumerate(order) if s == shape]
        ref = FBMEEngine(len(idx), shape[0], shape[1], cfg, dev, n_tile=eng.tile_widths[shape])
        ys = torch.stack([torch.from_numpy(sc[i].y).to(dev) for i in idx]).reshape(len(idx), -1)
        ref.run(ys.contiguous())
        torch.cuda.synchronize()
        n = shape[0][0] * shape[0][1]
        for j, i in enumerate(idx):
            p0 = eng.pix_off[i]
            for f in FIELDS_PIX:
                assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][j]), (f, i)
            for f in FIELDS_SCENE:
                assert torch.equal(eng.out[f][i], ref.out[f][j]), (f, i)
        ref.close()
    eng.close()


# FP32 FFT stages in uneven plans: every stage step is one merged two-pass
# FFT launch per transform length over the buckets of that length
FA = ((64, 64), (32, 32))
FB = ((128, 64), (48, 40))
FC = ((96, 128), (24, 64))
FD = ((512, 32), (200, 16))  # N1 = 512: adjoint stage 2 stores A^H m, the elementwise denoiser follows
F_ORDER = [FA, FB, FA, FC, FD, FB, FA]


def _fft_cfg(profile="stable"):
    from fbme_b200.config import fbme_profile_config

    cfg = fbme_profile_config(profile)
    cfg.dft_terms = -1  # automatic: every grid above allows the FFT stages
    return cfg


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
def test_fft_uneven_plan_equals_per_shape_plans(profile):
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    cfg = _fft_cfg(profile)
    sc = _scenes(F_ORDER, 900)
    eng = UnevenEngine(F_ORDER, cfg, dev)
    assert int(eng.native_cfg.dft_terms) == 0
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert len({b["uamp_iterations"] for b in eng.buckets()}) > 1
    for shape in (FA, FB, FC, FD):
        idx = [i for i, s in enumerate(F_ORDER) if s == shape]
        ref = FBMEEngine(len(idx), shape[0], shape[1], cfg, dev)
        assert int(ref.native_cfg.dft_terms) == 0
        ys = torch.stack([torch.from_numpy(sc[i].y).to(dev) for i in idx]).reshape(len(idx), -1)
        ref.run(ys.contiguous())
        torch.cuda.synchronize()
        n = shape[0][0] * shape[0][1]
        for j, i in enumerate(idx):
            p0 = eng.pix_off[i]
            for f in FIELDS_PIX:
                assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][j]), (f, i)
            for f in FIELDS_SCENE:
                assert torch.equal(eng.out[f][i], ref.out[f][j]), (f, i)
        ref.close()
    assert int(eng.out["status"].abs().sum()) == 0
    eng.close()


@pytest.mark.gpu
def test_fft_buckets_beyond_one_merged_launch():
    """70 shapes sharing N2 = 64: the N2-axis FFT steps hold 70 buckets of
    one length and split into two launches; every checked scene equals its
    single-scene FFT plan bit for bit."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(47)
    shapes = []
    while len(shapes) < 70:
        g = (int(rng.choice([32, 48, 64, 96])), 64)
        s = (int(rng.integers(8, g[0] // 2 + 1)), int(rng.integers(8, 33)))
        if (g, s) not in shapes:
            shapes.append((g, s))
    sc = _scenes(shapes, 3100)
    cfg = _fft_cfg()
    eng = UnevenEngine(shapes, cfg, dev)
    assert int(eng.native_cfg.dft_terms) == 0
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert len(eng.buckets()) == 70
    assert int(eng.out["status"].abs().sum()) == 0
    for i in range(0, 70, 3):
        g, s = shapes[i]
        ref = FBMEEngine(1, g, s, cfg, dev)
        ref.run(torch.from_numpy(sc[i].y).to(dev).reshape(1, -1).contiguous())
        torch.cuda.synchronize()
        p0, n = eng.pix_off[i], g[0] * g[1]
        for f in FIELDS_PIX:
            assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][0]), (f, i)
        for f in FIELDS_SCENE:
            assert torch.equal(eng.out[f][i], ref.out[f][0]), (f, i)
        ref.close()
    eng.close()


@pytest.mark.gpu
def test_fft_uneven_plan_with_short_transform_lengths():
    """Grids with 16- and 24-point axes take the FFT stages too (every length
    is 2^a or 3 * 2^a); lengths below the two-pass kernel's run one Stockham
    launch per bucket.  Every scene equals its equal-shape FFT plan bit for
    bit."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.uneven import UnevenEngine

    shapes = [((16, 32), (8, 16)), ((24, 48), (12, 20)), ((64, 16), (30, 8)), ((16, 32), (8, 16))]
    dev = torch.device("cuda", 0)
    cfg = _fft_cfg()
    cfg.uamp_polish_size = 32
    sc = _scenes(shapes, 4100)
    eng = UnevenEngine(shapes, cfg, dev)
    assert int(eng.native_cfg.dft_terms) == 0
    eng.run(eng.pack([torch.from_numpy(s.y).to(dev) for s in sc]))
    torch.cuda.synchronize()
    assert int(eng.out["status"].abs().sum()) == 0
    for i, (g, smp) in enumerate(shapes):
        ref = FBMEEngine(1, g, smp, cfg, dev)
        assert int(ref.native_cfg.dft_terms) == 0
        ref.run(torch.from_numpy(sc[i].y).to(dev).reshape(1, -1).contiguous())
        torch.cuda.synchronize()
        p0, n = eng.pix_off[i], g[0] * g[1]
        for f in FIELDS_PIX:
            assert torch.equal(eng.out[f][p0:p0 + n], ref.out[f][0]), (f, i)
        for f in FIELDS_SCENE:
            assert torch.equal(eng.out[f][i], ref.out[f][0]), (f, i)
        ref.close()
    eng.close()
