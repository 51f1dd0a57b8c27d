"""Pin the mode="cg" oracle against the reference and against known answers.

The fixtures in tests/golden/cg were produced by executing the reference
``fast_sbl(mode="cg", active_set=False)`` on the CPU in FP64 and FP32
(tests/golden/make_golden_cg.py).  The oracle's FP64 restatement must
reproduce the reference's FP64 run; the PCG restatement must solve SPD
Toeplitz systems with a known solution.
"""

import glob
from pathlib import Path

import numpy as np
import pytest

from oracle import fbme_oracle as O

CG = sorted(p for p in glob.glob(str(Path(__file__).parent / "golden" / "cg" / "cg_*.npz"))
            if not Path(p).name.startswith("cg_active_"))
ACTIVE = sorted(glob.glob(str(Path(__file__).parent / "golden" / "cg" / "cg_active_*.npz")))


def _rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("path", CG, ids=lambda p: Path(p).stem)
def test_cg_oracle_matches_reference_fp64(path):
    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    y = g["y"].astype(np.complex128)
    cfg = O.OracleConfig(mode="cg", active_set=False, max_iter=int(g["max_iter"]))
    r = O.fast_sbl_cg(y, grid, cfg, chol_mode="cpu")
    # dense reference fields are stored in single precision
    assert _rel(r["x"], g["f64_x"]) < 1e-6
    assert _rel(r["posterior_variance"], g["f64_posterior_variance"]) < 1e-5
    assert _rel(r["precision"], g["f64_precision"]) < 1e-6
    np.testing.assert_allclose(r["noise_variance"], g["f64_noise_variance"], rtol=1e-9)
    np.testing.assert_allclose(r["effective_dof"], g["f64_effective_dof"], rtol=1e-9)
    assert r["iterations"] == int(g["f64_iterations"])
    assert r["converged"] == bool(g["f64_converged"])
    np.testing.assert_array_equal(r["history"]["cg_iterations"], g["f64_history_cg_iterations"])
    np.testing.assert_allclose(r["history"]["relative_change"], g["f64_history_relative_change"],
                               rtol=1e-9)


@pytest.mark.parametrize("path", ACTIVE, ids=lambda p: Path(p).stem)
def test_cg_active_set_switch_matches_reference(path):
    """A single scene switches to the exact reduced posterior on the same
    ARD set at the same iteration as the reference (sbl_2d, mode="cg",
    default active-set parameters, CUDA Cholesky loading), and the FP64
    restatement reproduces the reference's FP64 run."""
    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    cfg = O.OracleConfig(mode="cg", max_iter=int(g["max_iter"]), tol=0.0)
    for tag, dtype, bar in (("f64", np.complex128, 1e-6), ("f32", np.complex64, 4.0 * float(g["gap_x"]))):
        r = O.fast_sbl_cg(g["y"][0].astype(dtype), grid, cfg)
        np.testing.assert_array_equal(r["history"]["active_set_size"], g[tag + "_history_active_set_size"])
        assert r["active_set_size"] == int(g[tag + "_active_set_size"])
        assert _rel(r["x"], g[tag + "_x"]) < bar
        assert _rel(r["posterior_variance"], g[tag + "_posterior_variance"]) < 1e2 * bar
        np.testing.assert_allclose(r["noise_variance"], g[tag + "_noise_variance"][0], rtol=1e2 * bar)
        np.testing.assert_allclose(r["effective_dof"], g[tag + "_effective_dof"][0], rtol=1e2 * bar)


DENSE = sorted(glob.glob(str(Path(__file__).parent / "golden" / "dense" / "dense_*.npz")))


@pytest.mark.parametrize("path", DENSE, ids=lambda p: Path(p).stem)
def test_dense_oracle_matches_reference_fp64(path):
    """mode="dense" (the exact posterior through the M x M data covariance)
    restated in FP64 reproduces the reference's FP64 run."""
    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    cfg = O.OracleConfig(mode="dense", max_iter=int(g["max_iter"]), tol=0.0)
    r = O.fast_sbl_dense(g["y"][0].astype(np.complex128), grid, cfg)
    assert r["mode"] == "dense"
    assert _rel(r["x"], g["f64_x"]) < 1e-6
    assert _rel(r["precision"], g["f64_precision"]) < 1e-6
    assert _rel(r["posterior_variance"], g["f64_posterior_variance"]) < 1e-5
    np.testing.assert_allclose(r["noise_variance"], g["f64_noise_variance"][0], rtol=1e-7)
    np.testing.assert_allclose(r["effective_dof"], g["f64_effective_dof"][0], rtol=1e-7)
    np.testing.assert_allclose(r["history"]["relative_change"], g["f64_history_relative_change"], rtol=1e-5)


def test_active_set_selection_rule():
    """solver.py:3184-3216 on hand-made priors: no switch while the tail
    holds more than the fraction, the smallest prefix reaching 1 - tail
    otherwise, clamped to [minimum, maximum]; batches never switch."""
    p = np.full((1, 100), 1e-3, np.float32)
    p[0, [5, 17, 42]] = [10.0, 5.0, 1.0]
    # total 16.097: 95 % needs the three large values, 90 % two of them
    np.testing.assert_array_equal(O.select_active_indices(p, 2, 10, 0.05), [[5, 17, 42]])
    np.testing.assert_array_equal(O.select_active_indices(p, 1, 10, 0.1), [[5, 17]])
    assert O.select_active_indices(p, 4, 10, 0.1).shape == (1, 4)
    # the 10 largest hold 16.007 < 99.9 % of the total: no switch
    assert O.select_active_indices(p, 1, 10, 0.001) is None
    flat = np.ones((1, 100), np.float32)
    assert O.select_active_indices(flat, 2, 10, 0.05) is None
    assert O.select_active_indices(np.concatenate([p, p]), 2, 10, 0.05) is None
    bad = p.copy()
    bad[0, 3] = np.nan
    assert O.select_active_indices(bad, 2, 10, 0.05) is None


def _dense_q(op, prior, noise):
    """Q = noise I + A diag(prior) A^H for one scene, FP64."""
    eye = np.eye(op.n_samples, dtype=np.complex128)[None]
    cols = op.adjoint(eye)[0]                      # A^H e_m, [N, M]
    a = np.conj(cols.T)                            # A, [M, N]
    return noise * np.eye(op.n_samples) + (a * prior[None, :]) @ np.conj(a.T)


def test_pcg_solves_toeplitz_system_with_known_solution():
    rng = np.random.default_rng(7)
    grid, sample = (24, 20), (10, 12)
    op = O.PrefixOperator(grid, sample, np.complex128)
    prior = rng.uniform(0.05, 1.0, (1, op.n_grid)) * np.where(rng.random((1, op.n_grid)) < 0.05, 50, 1)
    noise = np.array([0.2])
    x_true = rng.normal(size=(1, op.n_samples, 3)) + 1j * rng.normal(size=(1, op.n_samples, 3))
    q = _dense_q(op, prior[0], noise[0])
    rhs = (q @ x_true[0])[None]
    cfg = O.OracleConfig(cg_max_iter=150, cg_check_interval=8, cg_preconditioner_rank=8)
    x, it = O.pcg(rhs, prior, noise, op, cfg, initial=None, tolerance=1e-11, chol_mode="cpu")
    assert _rel(x, x_true) < 1e-8
    assert it < 150
    # the BTTB matvec and the Fourier matvec are the same matrix
    spec = op.toeplitz_spectrum(prior, noise)
    v = rng.normal(size=(1, op.n_samples, 2)) + 1j * rng.normal(size=(1, op.n_samples, 2))
    tbt = op.toeplitz_matvec(v, spec)
    four = noise[:, None, None] * v + op.forward(prior[:, :, None] * op.adjoint(v))
    assert _rel(tbt, four) < 1e-12
    assert _rel(four[0], q @ v[0]) < 1e-12


def test_pcg_fixed_iterations_keeps_best_checkpoint():
    rng = np.random.default_rng(3)
    op = O.PrefixOperator((16, 16), (8, 8), np.complex128)
    prior = rng.uniform(0.01, 1.0, (1, op.n_grid))
    noise = np.array([0.05])
    rhs = rng.normal(size=(1, op.n_samples, 2)) + 1j * rng.normal(size=(1, op.n_samples, 2))
    cfg = O.OracleConfig(cg_max_iter=40, cg_check_interval=4, cg_fixed_iterations=12)
    x, it = O.pcg(rhs, prior, noise, op, cfg, initial=None, tolerance=1e-14, chol_mode="cpu")
    assert it == 12
    q = _dense_q(op, prior[0], noise[0])
    res = np.linalg.norm(rhs[0] - q @ x[0], axis=0) / np.linalg.norm(rhs[0], axis=0)
    assert np.all(res < 1e-3)


def test_relevance_projection_caps_dof():
    prior = np.full((2, 50), 1.0)
    dd = np.full((2, 50), 0.9)
    rel = O.project_relevance(prior, dd, 20, np.finfo(np.float64).eps)
    assert np.all(rel.sum(axis=1) <= 20 * (1 - 10 * np.finfo(np.float64).eps) + 1e-9)
    assert np.all(rel <= 1.0) and np.all(rel >= 0.0)
