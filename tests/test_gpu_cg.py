"""mode="cg" (PCG + Hutchinson) on the B200 against the reference and the oracle.

Checkers:
  * the FP64 numpy oracle for the matvec and the PCG stage
    (fbme_cg_matvec, fbme_pcg_solve), including a dense FP64 solve;
  * golden vectors of the reference itself (tests/golden/cg, FP64 and FP32
    runs of ``fast_sbl(mode="cg", active_set=False)``) for the whole solve.

Tolerances.  PCG stops at a relative residual of max(cg_tolerance,
3 sqrt(eps_f32)) = 1.04e-3 in single precision, and the EM iteration
amplifies that difference: the reference's own FP32 run differs from its
FP64 run by the "gap" stored in each fixture (x: 6e-5 .. 4e-4 relative L2).
The device run (FP32 data, FP64 inner products) must stay within three
times that gap of the reference's FP64 run (x, precision), with the same
iteration count and the same 40 strongest coefficients per scene.  The
posterior variance comes from the Hutchinson diagonal of PCG solutions
that stop at the FP32 residual floor, so its bar is five times that floor.
"""

import glob
from pathlib import Path

import numpy as np
import pytest

from gpu_util import need_gpu, rel_l2

torch = pytest.importorskip("torch")

from oracle import fbme_oracle as O  # noqa: E402

CG = sorted(p for p in glob.glob(str(Path(__file__).parent / "golden" / "cg" / "cg_*.npz"))
            if not Path(p).name.startswith("cg_active_"))
ACTIVE = sorted(glob.glob(str(Path(__file__).parent / "golden" / "cg" / "cg_active_*.npz")))
PCG_FLOOR_F32 = 3.0 * float(np.finfo(np.float32).eps) ** 0.5  # solver.py:1349-1352


def _engine(batch, grid, sample, **kw):
    from fbme_b200.cg import CGEngine
    from fbme_b200.config import SBLConfig

    cfg = SBLConfig(mode="cg", active_set=False, **kw)
    return CGEngine(batch, grid, sample, cfg, torch.device("cuda"))


def _init_state(y, grid):
    """Initial prior / noise of the solver (solver.py:1063-1159), FP64."""
    b = y.shape[0]
    op = O.PrefixOperator(grid, y.shape[1:], np.complex128)
    yf = y.reshape(b, -1).astype(np.complex128)
    dp = np.maximum(np.mean(np.abs(yf) ** 2, axis=1), np.finfo(np.float32).eps)
    bp = op.adjoint_flat(yf)
    e = np.abs(bp) ** 2
    prior = 0.1 * e / e.sum(axis=1, keepdims=True) * dp[:, None] + 0.9 * dp[:, None] / op.n_grid
    prior = np.maximum(prior, dp[:, None] * 1e-12)
    noise = 0.01 * dp
    return op, prior, noise


def _dense_q(op, prior, noise):
    eye = np.eye(op.n_samples, dtype=np.complex128)[None]
    a = np.conj(op.adjoint(eye)[0].T)
    return noise * np.eye(op.n_samples) + (a * prior[None, :]) @ np.conj(a.T)


@pytest.mark.gpu
@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("grid,sample", [((64, 64), (32, 32)), ((48, 40), (20, 24))])
def test_cg_matvec_matches_fp64(terms, grid, sample):
    """Q v within 2e-5 relative L2 of FP64 (the DFT bar: FP32 tensor-core
    accumulation, measured 2-9e-6)."""
    need_gpu()
    rng = np.random.default_rng(11)
    B, R = 2, 3
    op = O.PrefixOperator(grid, sample, np.complex128)
    M = op.n_samples
    prior = rng.uniform(0.01, 1.0, (B, op.n_grid)) * np.where(rng.random((B, op.n_grid)) < 0.02, 30, 1)
    noise = rng.uniform(0.1, 0.5, B)
    v = rng.normal(size=(B, R, M)) + 1j * rng.normal(size=(B, R, M))
    ref = noise[:, None, None] * v + np.swapaxes(
        op.forward(prior[:, :, None] * op.adjoint(np.swapaxes(v, 1, 2))), 1, 2)
    eng = _engine(B, grid, sample, cg_dft_terms=terms)
    out = eng.matvec(torch.from_numpy(prior.astype(np.float32)).cuda(),
                     torch.from_numpy(noise.astype(np.float32)).cuda(),
                     torch.from_numpy(v.astype(np.complex64)).cuda())
    eng.close()
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


@pytest.mark.gpu
def test_pcg_matches_dense_solve_and_oracle_iterations():
    need_gpu()
    from scenes_util import c1_scene

    y, grid = c1_scene(0)
    op, prior, noise = _init_state(y[None], grid)
    M = op.n_samples
    probes = O.rademacher_probes(1, M, 4, 0)
    rhs = np.concatenate([y.reshape(1, M, 1), probes], axis=2).astype(np.complex128)  # [1, M, R]
    q = _dense_q(op, prior[0], noise[0])
    tol = 1e-4
    eng = _engine(1, grid, y.shape, cg_max_iter=150, cg_check_interval=8)
    x, it = eng.pcg(torch.from_numpy(prior.astype(np.float32)).cuda(),
                    torch.from_numpy(noise.astype(np.float32)).cuda(),
                    torch.from_numpy(np.swapaxes(rhs, 1, 2).astype(np.complex64)).cuda(), tol)
    eng.close()
    xs = np.swapaxes(x.cpu().numpy().astype(np.complex128), 1, 2)[0]  # [M, R]
    res = np.linalg.norm(rhs[0] - q @ xs, axis=0) / np.linalg.norm(rhs[0], axis=0)
    assert np.all(res < 1.5 * tol), res
    cfg = O.OracleConfig(cg_max_iter=150, cg_check_interval=8)
    _, it_o = O.pcg(rhs, prior, noise, op, cfg, initial=None, tolerance=tol, chol_mode="cuda")
    assert abs(it - it_o) <= 8, (it, it_o)


@pytest.mark.gpu
def test_pcg_fixed_iterations_matches_fp64_oracle():
    need_gpu()
    from scenes_util import c1_scene

    y, grid = c1_scene(1)
    op, prior, noise = _init_state(y[None], grid)
    M = op.n_samples
    rhs = np.concatenate([y.reshape(1, M, 1), O.rademacher_probes(1, M, 6, 2)], axis=2)
    rhs = rhs.astype(np.complex128)
    eng = _engine(1, grid, y.shape, cg_max_iter=150, cg_check_interval=8, cg_fixed_iterations=16)
    x, it = eng.pcg(torch.from_numpy(prior.astype(np.float32)).cuda(),
                    torch.from_numpy(noise.astype(np.float32)).cuda(),
                    torch.from_numpy(np.swapaxes(rhs, 1, 2).astype(np.complex64)).cuda(), 1e-6)
    eng.close()
    assert it == 16
    cfg = O.OracleConfig(cg_max_iter=150, cg_check_interval=8, cg_fixed_iterations=16)
    xo, _ = O.pcg(rhs, prior, noise, op, cfg, initial=None, tolerance=1e-6, chol_mode="cuda")
    assert rel_l2(np.swapaxes(x.cpu().numpy(), 1, 2), xo) < 5e-4


def _solve_golden(g, probes=None):
    grid = tuple(int(v) for v in g["grid"])
    y = g["y"]
    B, M = y.shape[0], y.shape[1] * y.shape[2]
    eng = _engine(B, grid, y.shape[1:], max_iter=int(g["max_iter"]))
    if probes is None:
        probes = O.rademacher_probes(B, M, eng.probes, 0)  # the reference's CPU stream
    z = torch.from_numpy(np.ascontiguousarray(np.swapaxes(probes, 1, 2)).astype(np.float32)).cuda()
    res = eng.solve(torch.from_numpy(y.reshape(B, M)).cuda(), z)
    eng.close()
    return res, probes


@pytest.mark.gpu
@pytest.mark.parametrize("path", CG, ids=lambda p: Path(p).stem)
def test_cg_solve_matches_reference_golden(path):
    need_gpu()
    g = np.load(path)
    res, _ = _solve_golden(g)
    B = g["y"].shape[0]
    x = res.x.cpu().numpy().reshape(B, -1)
    xr = g["f64_x"].reshape(B, -1)
    pv = res.posterior_variance.cpu().numpy().reshape(B, -1)
    prec = res.precision.cpu().numpy().reshape(B, -1)
    ex, epv, epr = rel_l2(x, xr), rel_l2(pv, g["f64_posterior_variance"]), rel_l2(prec, g["f64_precision"])
    print(f"{Path(path).stem}: x {ex:.2e} (ref gap {float(g['gap_x']):.2e}) pv {epv:.2e} "
          f"(ref gap {float(g['gap_posterior_variance']):.2e}) precision {epr:.2e}")
    assert ex < 3 * float(g["gap_x"]) + 2e-5
    # the Hutchinson variance inherits the PCG stopping residual (1.04e-3 in FP32)
    assert epv < max(3 * float(g["gap_posterior_variance"]), 5 * PCG_FLOOR_F32)
    assert epr < 3 * float(g["gap_precision"]) + 2e-5
    np.testing.assert_allclose(res.noise_variance.cpu().numpy().reshape(-1), g["f64_noise_variance"],
                               rtol=1e-3)
    np.testing.assert_allclose(res.effective_dof.cpu().numpy().reshape(-1), g["f64_effective_dof"],
                               rtol=1e-3)
    assert res.iterations == int(g["f64_iterations"])
    assert res.converged == bool(g["f64_converged"])
    for b in range(B):
        top = set(np.argsort(-np.abs(x[b]))[:40])
        top_r = set(np.argsort(-np.abs(xr[b]))[:40])
        assert top == top_r
    hist = np.asarray(res.history["cg_iterations"])
    assert np.mean(np.abs(hist - g["f64_history_cg_iterations"])) <= 8
    assert int(res.status.abs().sum()) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("path", ACTIVE, ids=lambda p: Path(p).stem)
def test_cg_active_set_switch_matches_reference_golden(path):
    """One scene with the default active-set switch (sbl_2d's defaults,
    tol=0, the reference's CPU probes): the switch comes at the reference's
    iteration with the reference's set size, and the result meets the bar
    of the cg fixtures against the reference's FP64 run."""
    need_gpu()
    from fbme_b200.cg import CGEngine
    from fbme_b200.config import SBLConfig

    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    y = g["y"]
    M = y.shape[1] * y.shape[2]
    cfg = SBLConfig(mode="cg", max_iter=int(g["max_iter"]), tol=0.0)
    eng = CGEngine(1, grid, y.shape[1:], cfg, torch.device("cuda"))
    probes = O.rademacher_probes(1, M, eng.probes, 0)
    z = torch.from_numpy(np.ascontiguousarray(np.swapaxes(probes, 1, 2)).astype(np.float32)).cuda()
    res = eng.solve(torch.from_numpy(y.reshape(1, M)).cuda(), z)
    eng.close()
    assert res.active_set_size == int(g["f64_active_set_size"])
    np.testing.assert_array_equal(res.history["active_set_size"], g["f64_history_active_set_size"])
    x = res.x.cpu().numpy().reshape(1, -1)
    ex = rel_l2(x, g["f64_x"].reshape(1, -1))
    epv = rel_l2(res.posterior_variance.cpu().numpy(), g["f64_posterior_variance"])
    epr = rel_l2(res.precision.cpu().numpy(), g["f64_precision"])
    print(f"{Path(path).stem}: x {ex:.2e} (ref gap {float(g['gap_x']):.2e}) pv {epv:.2e} "
          f"(ref gap {float(g['gap_posterior_variance']):.2e}) precision {epr:.2e}")
    assert ex < 3 * float(g["gap_x"]) + 2e-5
    assert epv < 3 * float(g["gap_posterior_variance"]) + 2e-5
    assert epr < 3 * float(g["gap_precision"]) + 2e-5
    np.testing.assert_allclose(res.noise_variance.cpu().numpy().reshape(-1), g["f64_noise_variance"],
                               rtol=1e-3)
    np.testing.assert_allclose(res.effective_dof.cpu().numpy().reshape(-1), g["f64_effective_dof"],
                               rtol=1e-3)
    assert res.iterations == int(g["f64_iterations"])
    assert int(res.status.abs().sum()) == 0


DENSE = sorted(glob.glob(str(Path(__file__).parent / "golden" / "dense" / "dense_*.npz")))


@pytest.mark.gpu
@pytest.mark.parametrize("path", DENSE, ids=lambda p: Path(p).stem)
def test_dense_mode_matches_reference_golden(path):
    """mode="dense" through sbl_2d against the reference's FP64 run: the
    device solves the data covariance in FP64 with the FP64 loading (the
    prior and the EM updates stay FP32 between iterations), so x, the
    precision, noise and DOF stay within a tenth of the reference's own
    FP32-FP64 gap, and the posterior variance, which the reference's FP32
    run loses to cancellation, matches its FP64 run."""
    need_gpu()
    from torch_sbl import SBLConfig, sbl_2d

    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    y = torch.from_numpy(g["y"][0]).cuda()
    res = sbl_2d(y, grid, config=SBLConfig(mode="dense", max_iter=int(g["max_iter"]), tol=0.0))
    assert res.mode == "dense" and res.iterations == int(g["f64_iterations"])
    ex = rel_l2(res.x.cpu().numpy(), g["f64_x"][0])
    epr = rel_l2(res.precision.cpu().numpy(), g["f64_precision"][0])
    epv = rel_l2(res.posterior_variance.cpu().numpy(), g["f64_posterior_variance"][0])
    print(f"{Path(path).stem}: x {ex:.2e} (ref FP32 gap {float(g['gap_x']):.2e}) precision {epr:.2e} "
          f"(gap {float(g['gap_precision']):.2e}) pv {epv:.2e} (gap {float(g['gap_posterior_variance']):.2e})")
    # the prior and the EM updates are FP32 between iterations: a tenth of
    # the reference's own FP32-FP64 gap
    assert ex < 0.1 * float(g["gap_x"])
    assert epr < 0.1 * float(g["gap_precision"])
    assert epv < 1e-3
    for f in ("noise_variance", "effective_dof"):
        ref64, ref32 = float(g["f64_" + f][0]), float(g["f32_" + f][0])
        got = float(getattr(res, f))
        print(f"  {f}: {got:.9g} (FP64 {ref64:.9g}, FP32 {ref32:.9g})")
        assert abs(got - ref64) <= 0.1 * abs(ref32 - ref64) + 1e-6 * abs(ref64)
    assert int(res.status.abs().sum()) == 0


@pytest.mark.gpu
def test_cg_batch_equals_single_scene_solves():
    need_gpu()
    g = np.load([p for p in CG if "_b2_" in p][0])
    res, probes = _solve_golden(g)
    for b in range(2):
        gb = {k: g[k] for k in g.files}
        gb["y"] = g["y"][b:b + 1]
        rb, _ = _solve_golden(gb, probes[b:b + 1])
        assert torch.equal(res.x.reshape(2, -1)[b], rb.x.reshape(-1))
        assert torch.equal(res.posterior_variance.reshape(2, -1)[b], rb.posterior_variance.reshape(-1))


@pytest.mark.gpu
def test_sbl_2d_cg_public_api():
    need_gpu()
    from scenes_util import c1_scene
    from torch_sbl import SBLConfig, sbl_2d

    y, grid = c1_scene(2)
    yt = torch.from_numpy(y).cuda()
    res = sbl_2d(yt, grid, config=SBLConfig(mode="cg", active_set=False, max_iter=6))
    assert res.mode == "cg" and res.x.shape == grid and res.iterations == 6
    assert np.isfinite(res.relative_change)
    assert len(res.history["cg_iterations"]) == 6 and res.uamp_backend_used is None
    # the reference's CUDA probe stream: same seed -> same result
    res2 = sbl_2d(yt, grid, config=SBLConfig(mode="cg", active_set=False, max_iter=6))
    assert torch.equal(res.x, res2.x)
    # the default single-scene call switches to the reduced posterior
    rd = sbl_2d(yt, grid, config=SBLConfig(mode="cg", max_iter=40))
    assert rd.active_set_size > 0 and rd.history["active_set_size"][-1] == rd.active_set_size
    assert rd.history["cg_iterations"][-1] == 0 and rd.history["hutchinson_probes"][-1] == 0
    batch = torch.stack([yt, yt])
    rb = sbl_2d(batch, grid, config=SBLConfig(mode="cg", max_iter=4,
                                               uamp_support_false_alarm_budget=0.5))
    assert rb.x.shape == (2, *grid) and rb.support_mask.shape == (2, *grid)


@pytest.mark.gpu
def test_cg_rank0_preconditioner_matches_oracle():
    need_gpu()
    from scenes_util import c1_scene

    y, grid = c1_scene(4)
    M = y.size
    eng = _engine(1, grid, y.shape, max_iter=5, cg_preconditioner_rank=0)
    probes = O.rademacher_probes(1, M, eng.probes, 0)
    z = torch.from_numpy(np.ascontiguousarray(np.swapaxes(probes, 1, 2)).astype(np.float32)).cuda()
    res = eng.solve(torch.from_numpy(y.reshape(1, M)).cuda(), z)
    eng.close()
    o = O.fast_sbl_cg(y[None].astype(np.complex128), grid,
                      O.OracleConfig(mode="cg", max_iter=5, cg_preconditioner_rank=0),
                      probes=probes, chol_mode="cuda")
    assert rel_l2(res.x.cpu().numpy().reshape(-1), o["x"].reshape(-1)) < 1e-3
