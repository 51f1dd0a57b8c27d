"""Golden vectors at the precision, batched-uneven and larger cg workloads,
made by executing the reference FBME-SBL package.

Run in a container that holds the reference source tree (it does not travel
to GPU machines); give its root in FBME_REFERENCE_ROOT:

    FBME_REFERENCE_ROOT=<path to FBME-SBL> python tests/golden/make_golden_configs.py

Cases (all solved by the reference on the CPU, ``uamp_backend="torch"``,
with the exact FBME-Stable / FBME-Fast plan configurations, as
make_golden.py does):

* ``c3_s{0,1,2}``: 512x512 grid, 256x192 prefix, 750 clustered + 50
  isolated log-normal points, 20 dB (``scenes.config_scene("c3", seed)``),
  in FP32 and FP64, with the reference's CUDA Cholesky loading, and the
  FP32 result's sensitivity to small input perturbations (make_c3).
* ``c4_b0``: the 64-scene batched-uneven workload of batch seed 0
  (``scenes.uneven_batch(0)``): grids from {128^2, 192x256, 256^2,
  384x256}, prefix ratios U[0.3, 0.7], 1-3 % CN(0,1) points, 5-25 dB,
  solved as the C3 scenes are (make_c4).  Per-scene
  results are packed with offsets.
* ``cg/cg_c2_s0_it6``: mode="cg" at 256x256 / 128x128 (``config_scene("c2",
  0)``), 6 EM iterations, FP64 and FP32 reference runs (format of
  make_golden_cg.py).
* ``cg/cg_active_c1_s0_it44``: one C1 scene through sbl_2d with mode="cg"
  and the default active-set switch, 44 iterations (make_cg_active).
* ``dense/dense_c1_s{0,1}_it30``: C1 scenes through sbl_2d with
  mode="dense", 30 iterations (make_dense).

The observations are not stored: the tests regenerate them with the
committed scene generator (numpy PCG64 streams, the same on every machine)
and check them against the SHA-256 stored here.
"""

from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]

PLAN_FIELDS = ("noise_variance", "effective_dof", "negative_log_evidence", "evidence_trace",
               "support_score_threshold", "fixed_budget_gamma_residual", "fixed_budget_noise_residual",
               "fixed_budget_objective_decrease", "fixed_budget_monotone", "support_exchanges_accepted")


def reference_root() -> str:
    root = os.environ.get("FBME_REFERENCE_ROOT")
    if not root or not (Path(root) / "torch_sbl" / "solver.py").exists():
        raise SystemExit("set FBME_REFERENCE_ROOT to the FBME-SBL source tree (holding torch_sbl/)")
    return root


def y_digest(y) -> str:
    import numpy as np

    return hashlib.sha256(np.ascontiguousarray(y, dtype=np.complex64).tobytes()).hexdigest()


def _import():
    sys.path.insert(0, reference_root())
    sys.path.append(str(REPO / "fbme-sbl_b200"))
    import torch
    from fbme_b200 import scenes
    from torch_sbl.solver import SBLConfig, fast_sbl  # reference package

    torch.set_num_threads(8)
    return torch, scenes, SBLConfig, fast_sbl


def plan_config(SBLConfig, profile: str):
    over = dict(device="cpu", uamp_backend="torch", uamp_polish_size=32,
                uamp_polish_compute_truncation_diagnostic=False)
    if profile == "stable":
        over.update(uamp_polish_iterations=3, uamp_polish_residual_exchange_size=12,
                    uamp_polish_fixed_budget_diagnostics=True)
    else:
        over.update(uamp_polish_iterations=2, uamp_polish_residual_exchange_size=0,
                    uamp_polish_fixed_budget_diagnostics=False)
    return SBLConfig.paper_hybrid_uamp(**over)


def _solve_fields(r, np):
    """Result fields of one reference solve, sparse where x is zero."""
    x = r.x.numpy().reshape(-1)
    act = np.flatnonzero(x != 0)
    pv = r.posterior_variance.numpy().reshape(-1)
    prec = r.precision.numpy().reshape(-1)
    inactive = np.ones(x.size, bool)
    inactive[act] = False
    out = {"active": act.astype(np.int64), "x_active": x[act], "pv_active": pv[act],
           "precision_active": prec[act], "pv_inactive_unique": np.unique(pv[inactive]),
           "precision_inactive_unique": np.unique(prec[inactive]),
           "mask_indices": np.flatnonzero(r.support_mask.numpy().reshape(-1)).astype(np.int64),
           "iterations": np.array(r.iterations)}
    for f in PLAN_FIELDS:
        v = getattr(r, f)
        if v is not None:
            out[f] = np.asarray(v.numpy())
    return out


def _cuda_cholesky_branch(S, torch):
    """The reference's CUDA branch of _stable_cholesky_raw (solver.py:2910-2920:
    one Cholesky with jitter_multiplier * eps * mean|diag| loading), run on
    the CPU tensors.  Its CPU branch tries 1 * eps first (2922-2931); on the
    ill-conditioned C3 reduced systems the two loadings give results that
    differ by more than the x parity bar, and the GPU replay takes this one."""

    def raw(matrix, identity, operator, *, sync_free_cholesky, jitter_multiplier, fallback_multipliers):
        scale = matrix.diagonal(dim1=-2, dim2=-1).real.abs().mean(dim=1)
        scale = scale.clamp_min(torch.finfo(operator.real_dtype).tiny)
        base = torch.finfo(matrix.real.dtype).eps * scale
        cand, info = torch.linalg.cholesky_ex(matrix + (jitter_multiplier * base)[:, None, None] * identity,
                                              check_errors=False)
        assert bool((info == 0).all()), "CUDA Cholesky branch failed"
        return cand

    return raw


# Relative size of the input perturbation that measures a scene's
# conditioning: 2^-17 (7.6e-6), the size of the device's split-BF16 DFT
# rounding (5-6e-6 relative L2 against an FP64 DFT).
PERTURBATION = 2.0 ** -17
PERTURBATION_DRAWS = 3


def _solve_three_ways(s, cfg, fast_sbl, torch, np):
    """One scene under one profile: FP32 fields, FP64 fields, the FP32-FP64
    gap, and the sensitivity: the largest change of the FP32 result (x in
    relative L2, posterior variance in max relative error on the support)
    over PERTURBATION_DRAWS inputs y * (1 + PERTURBATION * u), u ~ U[-1, 1]
    per real component, seeded."""
    r32 = fast_sbl(torch.from_numpy(s.y), s.grid, config=cfg)
    r64 = fast_sbl(torch.from_numpy(s.y.astype(np.complex128)), s.grid, config=cfg)
    x32, x64 = r32.x.numpy().ravel(), r64.x.numpy().ravel()
    v32, v64 = r32.posterior_variance.numpy().ravel(), r64.posterior_variance.numpy().ravel()
    a32, a64 = x32 != 0, x64 != 0
    gap_x = np.linalg.norm(x32 - x64) / np.linalg.norm(x64)
    gap_pv = np.max(np.abs(v32[a64] - v64[a64]) / v64[a64])
    sens_x = sens_pv = 0.0
    for k in range(PERTURBATION_DRAWS):
        rng = np.random.default_rng(1000 + k)
        u = rng.uniform(-1.0, 1.0, s.y.shape) + 1j * rng.uniform(-1.0, 1.0, s.y.shape)
        yp = (s.y.real.astype(np.float64) * (1 + PERTURBATION * u.real)
              + 1j * s.y.imag.astype(np.float64) * (1 + PERTURBATION * u.imag)).astype(np.complex64)
        rp = fast_sbl(torch.from_numpy(yp), s.grid, config=cfg)
        xp, vp = rp.x.numpy().ravel(), rp.posterior_variance.numpy().ravel()
        assert np.array_equal(xp != 0, a32), "a perturbation changed the support"
        sens_x = max(sens_x, float(np.linalg.norm(xp - x32) / np.linalg.norm(x32)))
        sens_pv = max(sens_pv, float(np.max(np.abs(vp[a32] - v32[a32]) / v32[a32])))
    return _solve_fields(r32, np), _solve_fields(r64, np), {"gap_x": gap_x, "gap_pv": gap_pv,
                                                             "sens_x": sens_x, "sens_pv": sens_pv}


def make_c3(seed: int) -> None:
    """C3 scene solved by the reference with its CUDA Cholesky loading:
    FP32 (``<profile>_*``, the replay's arithmetic; the parity target), FP64
    (``f64_<profile>_*``), their gap, and the FP32 result's sensitivity to
    input perturbations of the DFT rounding's size (``sens_<profile>_x``,
    ``sens_<profile>_pv``; _solve_three_ways).  The clustered scenes are
    ill-conditioned: their 32-atom reduced systems hold atoms one pixel
    apart, and the reference's own result moves by 5e-5 to 5e-3 under such
    perturbations, with the support unchanged."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene("c3", seed)
    out = {"grid": np.array(sc.grid), "sample": np.array(sc.y.shape), "y_sha256": np.array(y_digest(sc.y)),
           "scene": np.array(f"config_scene('c3', {seed})"), "x_true": sc.x.astype(np.complex64),
           "cholesky": np.array("cuda")}
    for profile in ("stable", "fast"):
        f32, f64, m = _solve_three_ways(sc, plan_config(SBLConfig, profile), fast_sbl, torch, np)
        for k, v in f32.items():
            out[profile + "_" + k] = v
        for k, v in f64.items():
            out["f64_" + profile + "_" + k] = v
        for k, v in m.items():
            a, b = k.split("_")
            out[f"{a}_{profile}_{b}"] = np.array(v)
    np.savez_compressed(HERE / f"c3_s{seed}.npz", **out)
    print("wrote", f"c3_s{seed}")


def make_c4(batch_seed: int) -> None:
    """All 64 scenes of one uneven batch, solved like make_c3.  Some of these
    scenes are ill-conditioned too (sensitivity up to ~3e-4).  Per-scene
    fields are concatenated, with offsets ``<field>_off``."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    batch = scenes.uneven_batch(batch_seed)
    out = {"grids": np.array([s.grid for s in batch], np.int64),
           "samples": np.array([s.y.shape for s in batch], np.int64),
           "y_sha256": np.array([y_digest(s.y) for s in batch]),
           "scene": np.array(f"uneven_batch({batch_seed})"), "cholesky": np.array("cuda")}
    for profile in ("stable", "fast"):
        cfg = plan_config(SBLConfig, profile)
        runs = [_solve_three_ways(s, cfg, fast_sbl, torch, np) for s in batch]
        for prefix, j in ((profile, 0), ("f64_" + profile, 1)):
            per = [r[j] for r in runs]
            for k in per[0]:
                vals = [np.atleast_1d(p[k]).reshape(-1) for p in per]
                out[f"{prefix}_{k}"] = np.concatenate(vals)
                out[f"{prefix}_{k}_off"] = np.concatenate([[0], np.cumsum([v.size for v in vals])]).astype(np.int64)
        for k in runs[0][2]:
            a, b = k.split("_")
            out[f"{a}_{profile}_{b}"] = np.array([r[2][k] for r in runs])
            out[f"{a}_{profile}_{b}_off"] = np.arange(len(runs) + 1, dtype=np.int64)
    np.savez_compressed(HERE / f"c4_b{batch_seed}.npz", **out)
    print("wrote", f"c4_b{batch_seed}")


def observation_mask(kind: str, sample, seed: int):
    """The masks of the masked fixtures: "random" keeps each sample with
    probability 0.7 (seeded); "ellipse" keeps the samples inside the
    ellipse inscribed in the M1 x M2 block (a non-rectangular aperture)."""
    import numpy as np

    m1, m2 = sample
    if kind == "random":
        return np.random.default_rng(50_000 + seed).random((m1, m2)) < 0.7
    a = (np.arange(m1)[:, None] + 0.5) / m1 - 0.5
    b = (np.arange(m2)[None, :] + 0.5) / m2 - 0.5
    return (a / 0.5) ** 2 + (b / 0.5) ** 2 <= 1.0


def make_masked(config: str, seed: int, kind: str) -> None:
    """A scene solved through the reference's sbl_2d with an observation
    mask (solver.py:986-1021, the masked PrefixFourierOperator) under the
    FBME plan configurations, CUDA Cholesky loading, with the FP32 result's
    sensitivity (the perturbation of _solve_three_ways, observed samples
    only)."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene(config, seed)
    mask = observation_mask(kind, sc.y.shape, seed)
    tm = torch.from_numpy(mask)
    out = {"grid": np.array(sc.grid), "sample": np.array(sc.y.shape), "y_sha256": np.array(y_digest(sc.y)),
           "scene": np.array(f"config_scene('{config}', {seed})"), "mask": mask, "mask_kind": np.array(kind),
           "cholesky": np.array("cuda")}
    for profile in ("stable", "fast"):
        cfg = plan_config(SBLConfig, profile)
        r = S.sbl_2d(torch.from_numpy(sc.y), sc.grid, config=cfg, observation_mask=tm)
        f = _solve_fields(r, np)
        x0, v0 = r.x.numpy().ravel(), r.posterior_variance.numpy().ravel()
        a0 = x0 != 0
        sens_x = sens_pv = 0.0
        for k in range(PERTURBATION_DRAWS):
            rng = np.random.default_rng(1000 + k)
            u = rng.uniform(-1.0, 1.0, sc.y.shape) + 1j * rng.uniform(-1.0, 1.0, sc.y.shape)
            yp = (sc.y.real.astype(np.float64) * (1 + PERTURBATION * u.real)
                  + 1j * sc.y.imag.astype(np.float64) * (1 + PERTURBATION * u.imag)).astype(np.complex64)
            rp = S.sbl_2d(torch.from_numpy(yp), sc.grid, config=cfg, observation_mask=tm)
            xp, vp = rp.x.numpy().ravel(), rp.posterior_variance.numpy().ravel()
            assert np.array_equal(xp != 0, a0), "a perturbation changed the support"
            sens_x = max(sens_x, float(np.linalg.norm(xp - x0) / np.linalg.norm(x0)))
            sens_pv = max(sens_pv, float(np.max(np.abs(vp[a0] - v0[a0]) / v0[a0])))
        for k, v in f.items():
            out[profile + "_" + k] = v
        out[f"sens_{profile}_x"] = np.array(sens_x)
        out[f"sens_{profile}_pv"] = np.array(sens_pv)
        out[f"{profile}_mode"] = np.array(r.mode)
    name = f"masked_{config}_{kind}_s{seed}"
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print("wrote", name)


def make_cg_c2(seed: int, max_iter: int) -> None:
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    sc = scenes.config_scene("c2", seed)
    y = sc.y[None]
    out = {"y": y, "grid": np.array(sc.grid), "seeds": np.array([seed]), "max_iter": np.array(max_iter),
           "x_true": sc.x[None].astype(np.complex64)}
    runs = {}
    for tag, dtype in (("f64", np.complex128), ("f32", np.complex64)):
        cfg = SBLConfig(mode="cg", active_set=False, max_iter=max_iter, device="cpu", return_history=True)
        r = fast_sbl(torch.from_numpy(y.astype(dtype)), sc.grid, config=cfg)
        runs[tag] = r
        if tag == "f64":
            out[tag + "_x"] = r.x.numpy().astype(np.complex64)
            out[tag + "_posterior_variance"] = r.posterior_variance.numpy().astype(np.float32)
            out[tag + "_precision"] = r.precision.numpy().astype(np.float32)
        out[tag + "_noise_variance"] = r.noise_variance.numpy()
        out[tag + "_effective_dof"] = r.effective_dof.numpy()
        out[tag + "_iterations"] = np.array(r.iterations)
        out[tag + "_converged"] = np.array(r.converged)
        out[tag + "_relative_change"] = np.array(r.relative_change)
        for key in ("relative_change", "noise_variance", "effective_dof", "cg_iterations",
                    "hutchinson_probes", "cg_tolerance"):
            out[tag + "_history_" + key] = np.array(r.history[key])

    def gap(a, b):
        a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    for f in ("x", "posterior_variance", "precision"):
        out["gap_" + f] = np.array(gap(getattr(runs["f32"], f).numpy(), getattr(runs["f64"], f).numpy()))
    (HERE / "cg").mkdir(exist_ok=True)
    name = f"cg_c2_s{seed}_it{max_iter}"
    np.savez_compressed(HERE / "cg" / f"{name}.npz", **out)
    print("wrote", name)


def make_dense(config: str, seed: int, max_iter: int) -> None:
    """A single scene through the reference's ``sbl_2d`` with
    ``mode="dense"`` (the exact posterior through the M x M data covariance,
    solver.py:2962-2990; what ``mode="auto"`` picks for M <= 2048), ``tol=0``,
    CUDA Cholesky loading; FP64 and FP32 runs in the cg fixture format."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene(config, seed)
    out = {"y": sc.y[None], "grid": np.array(sc.grid), "seeds": np.array([seed]),
           "max_iter": np.array(max_iter), "x_true": sc.x[None].astype(np.complex64),
           "cholesky": np.array("cuda"), "mode": np.array("dense")}
    runs = {}
    for tag, dtype in (("f64", np.complex128), ("f32", np.complex64)):
        cfg = SBLConfig(mode="dense", max_iter=max_iter, tol=0.0, device="cpu", return_history=True)
        r = S.sbl_2d(torch.from_numpy(sc.y.astype(dtype)), sc.grid, config=cfg)
        assert r.mode == "dense"
        runs[tag] = r
        out[tag + "_x"] = r.x.numpy().astype(np.complex64)[None]
        out[tag + "_posterior_variance"] = r.posterior_variance.numpy().astype(np.float32)[None]
        out[tag + "_precision"] = r.precision.numpy().astype(np.float32)[None]
        out[tag + "_noise_variance"] = np.atleast_1d(r.noise_variance.numpy())
        out[tag + "_effective_dof"] = np.atleast_1d(r.effective_dof.numpy())
        out[tag + "_iterations"] = np.array(r.iterations)
        for key in ("relative_change", "noise_variance", "effective_dof"):
            out[tag + "_history_" + key] = np.array(r.history[key])

    def gap(a, b):
        a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    for f in ("x", "posterior_variance", "precision"):
        out["gap_" + f] = np.array(gap(getattr(runs["f32"], f).numpy(), getattr(runs["f64"], f).numpy()))
    (HERE / "dense").mkdir(exist_ok=True)
    name = f"dense_{config}_s{seed}_it{max_iter}"
    np.savez_compressed(HERE / "dense" / f"{name}.npz", **out)
    print("wrote", name, "gaps", out["gap_x"], out["gap_posterior_variance"])


def make_cg_active(config: str, seed: int, max_iter: int) -> None:
    """A single scene through the reference's ``sbl_2d`` with ``mode="cg"``
    and its default active-set switch (solver.py:1316-1341: from iteration
    30, every 2 iterations, once at most 256 coefficients hold 95 % of the
    prior variance, the exact reduced posterior on them replaces PCG),
    ``tol=0`` so that every run takes ``max_iter`` iterations, with the
    reference's CUDA Cholesky loading; FP64 and FP32 runs, format of
    make_cg_c2 plus the active set."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene(config, seed)
    out = {"y": sc.y[None], "grid": np.array(sc.grid), "seeds": np.array([seed]),
           "max_iter": np.array(max_iter), "x_true": sc.x[None].astype(np.complex64),
           "cholesky": np.array("cuda")}
    runs = {}
    for tag, dtype in (("f64", np.complex128), ("f32", np.complex64)):
        cfg = SBLConfig(mode="cg", max_iter=max_iter, tol=0.0, device="cpu", return_history=True)
        r = S.sbl_2d(torch.from_numpy(sc.y.astype(dtype)), sc.grid, config=cfg)
        runs[tag] = r
        out[tag + "_x"] = r.x.numpy().astype(np.complex64)[None]
        out[tag + "_posterior_variance"] = r.posterior_variance.numpy().astype(np.float32)[None]
        out[tag + "_precision"] = r.precision.numpy().astype(np.float32)[None]
        out[tag + "_noise_variance"] = np.atleast_1d(r.noise_variance.numpy())
        out[tag + "_effective_dof"] = np.atleast_1d(r.effective_dof.numpy())
        out[tag + "_iterations"] = np.array(r.iterations)
        out[tag + "_active_set_size"] = np.array(r.active_set_size)
        for key in ("relative_change", "noise_variance", "effective_dof", "cg_iterations",
                    "hutchinson_probes", "cg_tolerance", "active_set_size"):
            out[tag + "_history_" + key] = np.array(r.history[key])

    def gap(a, b):
        a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    for f in ("x", "posterior_variance", "precision"):
        out["gap_" + f] = np.array(gap(getattr(runs["f32"], f).numpy(), getattr(runs["f64"], f).numpy()))
    (HERE / "cg").mkdir(exist_ok=True)
    name = f"cg_active_{config}_s{seed}_it{max_iter}"
    np.savez_compressed(HERE / "cg" / f"{name}.npz", **out)
    print("wrote", name, "active set", out["f32_active_set_size"], out["f64_active_set_size"])


CERT_FIELDS = ("inactive_max_evidence_ratio", "inactive_best_index", "inactive_evidence_gain",
               "inactive_optimal_variance", "support_repairs_accepted", "support_exchanges_accepted",
               "active_max_evidence_gain", "active_best_index", "active_optimal_variance",
               "active_max_deletion_gain", "coordinate_stationary", "inactive_ratio_threshold",
               "type2_coordinate_stationary", "stationarity_ratio_threshold", "familywise_ratio_threshold",
               "familywise_no_discovery", "familywise_support_certified", "inactive_penalized_evidence_gain",
               "active_penalized_evidence_gain", "type2_map_coordinate_stationary", "noise_variance",
               "effective_dof", "negative_log_evidence", "evidence_trace", "penalized_negative_log_evidence")


def make_certified(config: str, seed: int, repairs: int, fwer: float) -> None:
    """A scene solved by the reference's sbl_2d under certified_hybrid_uamp
    (global certificate, support repairs; solver.py:300-316), CUDA Cholesky
    loading; fwer > 0 adds the familywise screening threshold."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene(config, seed)
    over = dict(device="cpu", uamp_backend="torch", uamp_polish_compute_truncation_diagnostic=False,
                uamp_polish_support_repairs=repairs)
    if fwer > 0:
        over["uamp_polish_familywise_error_rate"] = fwer
    r = S.sbl_2d(torch.from_numpy(sc.y), sc.grid, config=SBLConfig.certified_hybrid_uamp(**over))
    x = r.x.numpy().reshape(-1)
    act = np.flatnonzero(x != 0)
    inactive = np.ones(x.size, bool)
    inactive[act] = False
    pv, prec = r.posterior_variance.numpy().reshape(-1), r.precision.numpy().reshape(-1)
    out = {"grid": np.array(sc.grid), "sample": np.array(sc.y.shape), "y_sha256": np.array(y_digest(sc.y)),
           "scene": np.array(f"config_scene('{config}', {seed})"), "repairs": np.array(repairs),
           "fwer": np.array(fwer), "cholesky": np.array("cuda"), "active": act.astype(np.int64),
           "x_active": x[act], "pv_active": pv[act], "precision_active": prec[act],
           "pv_inactive_unique": np.unique(pv[inactive]), "precision_inactive_unique": np.unique(prec[inactive])}
    for f in CERT_FIELDS:
        v = getattr(r, f)
        if v is not None:
            out[f] = np.asarray(v.numpy())
    name = f"cert_{config}_s{seed}_r{repairs}" + ("_fw" if fwer > 0 else "")
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print("wrote", name, "repairs kept", int(r.support_repairs_accepted))


JOBS = [("c3", "0"), ("c3", "1"), ("c3", "2"), ("c4", "0"), ("cg_c2", "0", "6"),
        ("masked", "c1", "0", "random"), ("masked", "c1", "1", "ellipse"), ("masked", "c2", "0", "random"),
        ("masked", "c2", "1", "ellipse"), ("cg_active", "c1", "0", "44"),
        ("dense", "c1", "0", "30"), ("dense", "c1", "1", "30"),
        ("certified", "c1", "0", "1", "0"), ("certified", "c2", "0", "1", "0"),
        ("certified", "c1", "1", "3", "0.05"), ("certified", "c2", "1", "2", "0")]


def main() -> None:
    if len(sys.argv) > 1:
        if sys.argv[1] == "masked":
            make_masked(sys.argv[2], int(sys.argv[3]), sys.argv[4])
            return
        if sys.argv[1] == "certified":
            make_certified(sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), float(sys.argv[5]))
            return
        if sys.argv[1] in ("cg_active", "dense"):
            {"cg_active": make_cg_active, "dense": make_dense}[sys.argv[1]](
                sys.argv[2], int(sys.argv[3]), int(sys.argv[4]))
            return
        kind, args = sys.argv[1], [int(v) for v in sys.argv[2:]]
        {"c3": make_c3, "c4": make_c4, "cg_c2": make_cg_c2}[kind](*args)
        return
    reference_root()
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    for job in JOBS:
        subprocess.run([sys.executable, __file__, *job], check=True, env=env)


if __name__ == "__main__":
    main()
