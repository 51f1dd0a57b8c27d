"""FBME-Stable / FBME-Fast plan replay on the B200 against the reference.

Two checkers:
  * the golden fixtures, i.e. outputs of the reference package itself
    (tests/golden, produced by tests/golden/make_golden.py);
  * the numpy oracle on freshly generated seeded scenes.
Bar: identical final support, x within 1e-4 relative L2, posterior variance
within 1e-3 relative on the support, noise / evidence within 1e-4 relative.
"""

import glob
from pathlib import Path

import numpy as np
import pytest

from gpu_util import PV_TOL, X_TOL, need_gpu, rel_l2

torch = pytest.importorskip("torch")

GOLDEN = sorted(glob.glob(str(Path(__file__).parent / "golden" / "*.npz")))


def _plan(profile, y, grid):
    from torch_sbl_fastest_stable import make_fastest_plan, make_stable_plan

    make = make_stable_plan if profile == "stable" else make_fastest_plan
    return make(y, grid, polish_size=32, warmup=1)


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: Path(p).stem)
def test_plan_matches_reference_golden(path, profile):
    need_gpu()
    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    y = torch.from_numpy(g["y"]).cuda()
    res = _plan(profile, y, grid).replay(y, synchronize=True)
    p = profile + "_"
    x = res.x.cpu().numpy().reshape(-1)
    act = np.flatnonzero(x)
    assert set(act) == set(g[p + "active"])
    xr = np.zeros_like(x)
    xr[g[p + "active"]] = g[p + "x_active"]
    assert rel_l2(x, xr) < X_TOL
    pv = res.posterior_variance.cpu().numpy().reshape(-1)
    np.testing.assert_allclose(pv[g[p + "active"]], g[p + "pv_active"], rtol=PV_TOL)
    np.testing.assert_allclose(res.noise_variance.cpu().numpy(), g[p + "noise_variance"], rtol=1e-4)
    np.testing.assert_allclose(res.negative_log_evidence.cpu().numpy(), g[p + "negative_log_evidence"],
                               rtol=1e-4)
    np.testing.assert_allclose(res.evidence_trace.cpu().numpy(), g[p + "evidence_trace"], rtol=1e-4)
    np.testing.assert_allclose(res.effective_dof.cpu().numpy(), g[p + "effective_dof"], rtol=1e-4)
    assert np.array_equal(np.flatnonzero(res.support_mask.cpu().numpy().reshape(-1)), g[p + "mask_indices"])
    assert res.iterations == int(g[p + "iterations"])
    assert int(res.status.item()) == 0
    if profile == "stable":
        assert int(res.support_exchanges_accepted.item()) == int(g[p + "support_exchanges_accepted"])
        assert bool(res.fixed_budget_monotone.item()) == bool(g[p + "fixed_budget_monotone"])
        np.testing.assert_allclose(res.fixed_budget_noise_residual.cpu().numpy(),
                                   g[p + "fixed_budget_noise_residual"], rtol=2e-2, atol=1e-6)
        np.testing.assert_allclose(res.fixed_budget_gamma_residual.cpu().numpy(),
                                   g[p + "fixed_budget_gamma_residual"], rtol=2e-2, atol=1e-6)
    else:
        assert res.fixed_budget_monotone is None and res.support_exchanges_accepted is None


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
