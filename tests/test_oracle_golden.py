"""Pin the numpy oracle against golden vectors from the reference itself.

The fixtures in tests/golden were produced by executing the reference
FBME-SBL ``fast_sbl`` (CPU, ``uamp_backend="torch"``) with the exact
FBME-Stable / FBME-Fast plan configurations (tests/golden/make_golden.py).
The oracle runs with the reference's CPU Cholesky loading schedule
(torch_sbl/solver.py:2922-2931) for this comparison.
"""

import glob

import numpy as np
import pytest

from oracle import fbme_oracle as O

FILES = sorted(glob.glob(str(__import__("pathlib").Path(__file__).parent / "golden" / "*.npz")))


@pytest.mark.parametrize("path", FILES, ids=lambda p: p.rsplit("/", 1)[-1][:-4])
@pytest.mark.parametrize("profile", ["stable", "fast"])
def test_oracle_matches_reference(path, profile):
    g = np.load(path)
    r = O.fbme_solve(g["y"], tuple(int(v) for v in g["grid"]), profile, chol_mode="cpu")
    p = profile + "_"
    x = r["x"].reshape(-1)
    act = np.flatnonzero(x != 0)
    # identical final active set (the support of x)
    assert np.array_equal(np.sort(act), np.sort(g[p + "active"]))
    xr = np.zeros_like(x)
    xr[g[p + "active"]] = g[p + "x_active"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 2e-5
    pv = r["posterior_variance"].reshape(-1)
    np.testing.assert_allclose(pv[g[p + "active"]], g[p + "pv_active"], rtol=1e-4)
    inactive = np.setdiff1d(np.arange(x.size), act)
    np.testing.assert_allclose(np.unique(pv[inactive]), g[p + "pv_inactive_unique"], rtol=1e-6)
    np.testing.assert_allclose(r["precision"].reshape(-1)[g[p + "active"]],
                               g[p + "precision_active"], rtol=1e-4)
    np.testing.assert_allclose(r["noise_variance"], g[p + "noise_variance"], rtol=1e-5)
    np.testing.assert_allclose(r["effective_dof"], g[p + "effective_dof"], rtol=1e-5)
    np.testing.assert_allclose(r["negative_log_evidence"], g[p + "negative_log_evidence"], rtol=1e-5)
    np.testing.assert_allclose(r["evidence_trace"], g[p + "evidence_trace"], rtol=1e-5)
    assert np.array_equal(np.flatnonzero(r["support_mask"].reshape(-1)), g[p + "mask_indices"])
    assert r["iterations"] == int(g[p + "iterations"])
    if profile == "stable":
        assert int(r["support_exchanges_accepted"]) == int(g[p + "support_exchanges_accepted"])
        np.testing.assert_allclose(r["fixed_budget_noise_residual"],
                                   g[p + "fixed_budget_noise_residual"], rtol=1e-3, atol=1e-7)
        np.testing.assert_allclose(r["fixed_budget_gamma_residual"],
                                   g[p + "fixed_budget_gamma_residual"], rtol=2e-3, atol=1e-7)
        assert bool(r["fixed_budget_monotone"]) == bool(g[p + "fixed_budget_monotone"])
