"""FBME-Stable / FBME-Fast plan replay on the B200 against the reference.

Two checkers:
  * the golden fixtures, i.e. outputs of the reference package itself
    (tests/golden, produced by tests/golden/make_golden.py);
  * the numpy oracle on freshly generated seeded scenes.
Bar: identical final support, x within 1e-4 relative L2, posterior variance
within 1e-3 relative on the support, noise / evidence within 1e-4 relative.
"""

from pathlib import Path

import numpy as np
import pytest

from golden_util import (PLAN_FILES, SENS_FACTOR, UNEVEN_FILES, plan_case, scene_fields, sensitivity,
                         uneven_case)
from gpu_util import PV_TOL, X_TOL, need_gpu, rel_l2

torch = pytest.importorskip("torch")


def _plan(profile, y, grid):
    from torch_sbl_fastest_stable import make_fastest_plan, make_stable_plan

    make = make_stable_plan if profile == "stable" else make_fastest_plan
    return make(y, grid, polish_size=32, warmup=1)


def _check_plan_fields(res, g, profile, sens=(0.0, 0.0), label=""):
    """One scene's plan result against a reference fixture's fields.  On an
    ill-conditioned scene (sens = the reference's own sensitivity, see
    golden_util.SENS_FACTOR) the value bars widen to SENS_FACTOR * sens."""
    p = profile + "_"
    sel = lambda t: t.cpu().numpy().reshape(-1)  # noqa: E731
    x_tol, pv_tol = max(X_TOL, SENS_FACTOR * sens[0]), max(PV_TOL, SENS_FACTOR * sens[1])
    s_tol = max(1e-4, SENS_FACTOR * sens[0])
    x = sel(res.x)
    act = np.flatnonzero(x)
    assert set(act) == set(g[p + "active"]), label
    xr = np.zeros_like(x)
    xr[g[p + "active"]] = g[p + "x_active"]
    err = rel_l2(x, xr)
    if sens[0] > 0:
        print(f"{label} {profile}: x {err:.2e} (bar {x_tol:.2e}, reference sensitivity {sens[0]:.2e})")
    assert err < x_tol, (label, err, x_tol)
    pv = sel(res.posterior_variance)
    np.testing.assert_allclose(pv[g[p + "active"]], g[p + "pv_active"], rtol=pv_tol, err_msg=label)
    for f in ("noise_variance", "negative_log_evidence", "evidence_trace", "effective_dof"):
        np.testing.assert_allclose(sel(getattr(res, f)), np.reshape(g[p + f], -1), rtol=s_tol, err_msg=label + f)
    assert np.array_equal(np.flatnonzero(sel(res.support_mask)), g[p + "mask_indices"]), label
    assert int(sel(res.status)[0]) == 0, label
    assert res.iterations == int(np.reshape(g[p + "iterations"], -1)[0]), label
    if profile == "stable":
        assert int(sel(res.support_exchanges_accepted)[0]) == int(g[p + "support_exchanges_accepted"]), label
        assert bool(sel(res.fixed_budget_monotone)[0]) == bool(g[p + "fixed_budget_monotone"]), label
        for f in ("fixed_budget_noise_residual", "fixed_budget_gamma_residual"):
            dev, ref = float(sel(getattr(res, f))[0]), float(np.reshape(g[p + f], -1)[0])
            print(f"{label} {f}: device {dev:.7g} reference {ref:.7g} rel {abs(dev - ref) / abs(ref):.2e}")
            np.testing.assert_allclose(dev, ref, rtol=2e-2, atol=1e-6, err_msg=label + f)
    else:
        assert res.fixed_budget_monotone is None and res.support_exchanges_accepted is None


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
@pytest.mark.parametrize("path", PLAN_FILES, ids=lambda p: Path(p).stem)
def test_plan_matches_reference_golden(path, profile):
    need_gpu()
    y_np, grid, g = plan_case(path)
    y = torch.from_numpy(y_np).cuda()
    res = _plan(profile, y, grid).replay(y, synchronize=True)
    _check_plan_fields(res, g, profile, sensitivity(g, profile), label=Path(path).stem)


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
@pytest.mark.parametrize("path", UNEVEN_FILES, ids=lambda p: Path(p).stem)
def test_uneven_plan_matches_reference_golden(path, profile):
    """The 64-scene batched-uneven workload (four grids, prefix ratios in
    [0.3, 0.7]) in one uneven plan against the reference's per-scene solves."""
    need_gpu()
    from fbme_b200.uneven import make_uneven_plan

    batch, g = uneven_case(path)
    ys = [torch.from_numpy(s.y).cuda() for s in batch]
    plan = make_uneven_plan(ys, [s.grid for s in batch], profile=profile, polish_size=32, warmup=1)
    results = plan.replay(ys, synchronize=True)
    assert len(results) == len(batch)
    for i, r in enumerate(results):
        _check_plan_fields(r, scene_fields(g, profile, i), profile, sensitivity(g, profile, i),
                           label=f"scene {i} {batch[i].grid}/{batch[i].y.shape}")


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
def test_batched_plan_matches_oracle(profile):
    """Eight C2 scenes in one plan (leading batch dimension) vs the oracle."""
    need_gpu()
    from fbme_b200 import scenes
    from oracle import fbme_oracle as O

    sc = [scenes.config_scene("c2", 100 + i) for i in range(8)]
    y_np = np.stack([s.y for s in sc])
    y = torch.from_numpy(y_np).cuda()
    res = _plan(profile, y, (256, 256)).replay(y, synchronize=True)
    ref = O.fbme_solve(y_np, (256, 256), profile)
    x = res.x.cpu().numpy().reshape(8, -1)
    xr = ref["x"].reshape(8, -1)
    for i in range(8):
        assert set(np.flatnonzero(x[i])) == set(np.flatnonzero(xr[i]))
        assert rel_l2(x[i], xr[i]) < X_TOL
    pv = res.posterior_variance.cpu().numpy().reshape(8, -1)
    pvr = ref["posterior_variance"].reshape(8, -1)
    sup = xr != 0
    assert np.max(np.abs(pv[sup] - pvr[sup]) / pvr[sup]) < PV_TOL
    np.testing.assert_allclose(res.noise_variance.cpu().numpy(), ref["noise_variance"], rtol=1e-4)
    assert int(res.status.abs().sum()) == 0


@pytest.mark.gpu
def test_batch_equals_single_scene_bitwise():
    """Scenes are independent: a scene's result does not depend on its batch."""
    need_gpu()
    from fbme_b200 import scenes

    sc = [scenes.config_scene("c1", i) for i in range(5)]
    y = torch.from_numpy(np.stack([s.y for s in sc])).cuda()
    rb = _plan("stable", y, (64, 64)).replay(y, synchronize=True)
    xb = rb.x.clone()
    for i in (0, 3):
        ri = _plan("stable", y[i].contiguous(), (64, 64)).replay(y[i].contiguous(), synchronize=True)
        assert torch.equal(ri.x, xb[i])


@pytest.mark.gpu
def test_replays_are_bit_reproducible_and_graph_owned():
    need_gpu()
    from fbme_b200 import scenes

    s0, s1 = scenes.config_scene("c1", 0), scenes.config_scene("c1", 1)
    y0 = torch.from_numpy(s0.y).cuda()
    y1 = torch.from_numpy(s1.y).cuda()
    plan = _plan("stable", y0, (64, 64))
    r = plan.replay(y0, synchronize=True)
    a = r.x.clone()
    r1 = plan.replay(y1, synchronize=True)
    assert r1 is plan.result and r1.x.data_ptr() == r.x.data_ptr()  # graph-owned
    assert not torch.equal(r1.x, a)
    r2 = plan.replay(y0, synchronize=True)
    assert torch.equal(r2.x, a)  # deterministic reductions


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
@pytest.mark.parametrize("path", [p for p in PLAN_FILES if "rtx_" not in p], ids=lambda p: Path(p).stem)
def test_fp32_fft_mode_plan_matches_reference_golden(path, profile):
    """The plans with the operator as FP32 FFTs (dft_terms=0) meet the same
    bar against the reference."""
    need_gpu()
    from fbme_b200.config import fbme_profile_config
    from fbme_b200.plans import CUDAGraphSBLPlan

    y_np, grid, g = plan_case(path)
    y = torch.from_numpy(y_np).cuda()
    cfg = fbme_profile_config(profile)
    cfg.dft_terms = 0
    res = CUDAGraphSBLPlan(y, grid, config=cfg, warmup=1).replay(y, synchronize=True)
    _check_plan_fields(res, g, profile, sensitivity(g, profile), label=Path(path).stem + " fft")
