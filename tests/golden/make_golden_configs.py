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
  in FP32 and FP64, with the reference's CUDA Cholesky loading (make_c3).
* ``c4_b0``: the 64-scene batched-uneven workload of batch seed 0
  (``scenes.uneven_batch(0)``): grids from {128^2, 192x256, 256^2,
  384x256}, prefix ratios U[0.3, 0.7], 1-3 % CN(0,1) points, 5-25 dB.
  Per-scene results are packed with offsets.
* ``cg/cg_c2_s0_it6``: mode="cg" at 256x256 / 128x128 (``config_scene("c2",
  0)``), 6 EM iterations, FP64 and FP32 reference runs (format of
  make_golden_cg.py).

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


def make_c3(seed: int) -> None:
    """C3 scene solved three ways by the reference, all with its CUDA
    Cholesky loading: FP32 (``<profile>_*``, the replay's arithmetic), FP64
    (``f64_<profile>_*``, complex128 input promotes the whole pipeline) and
    their gap, which measures how far the reference's own FP32 result sits
    from the exact one on this ill-conditioned scene."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    import torch_sbl.solver as S  # reference package

    S._stable_cholesky_raw = _cuda_cholesky_branch(S, torch)
    sc = scenes.config_scene("c3", seed)
    out = {"grid": np.array(sc.grid), "sample": np.array(sc.y.shape), "y_sha256": np.array(y_digest(sc.y)),
           "scene": np.array(f"config_scene('c3', {seed})"), "x_true": sc.x.astype(np.complex64),
           "cholesky": np.array("cuda")}
    for profile in ("stable", "fast"):
        cfg = plan_config(SBLConfig, profile)
        r32 = fast_sbl(torch.from_numpy(sc.y), sc.grid, config=cfg)
        r64 = fast_sbl(torch.from_numpy(sc.y.astype(np.complex128)), sc.grid, config=cfg)
        for k, v in _solve_fields(r32, np).items():
            out[profile + "_" + k] = v
        for k, v in _solve_fields(r64, np).items():
            out["f64_" + profile + "_" + k] = v
        x32, x64 = r32.x.numpy().ravel(), r64.x.numpy().ravel()
        out["gap_" + profile + "_x"] = np.array(np.linalg.norm(x32 - x64) / np.linalg.norm(x64))
        v32, v64 = r32.posterior_variance.numpy().ravel(), r64.posterior_variance.numpy().ravel()
        act = x64 != 0
        out["gap_" + profile + "_pv"] = np.array(np.max(np.abs(v32[act] - v64[act]) / v64[act]))
    np.savez_compressed(HERE / f"c3_s{seed}.npz", **out)
    print("wrote", f"c3_s{seed}")


def make_c4(batch_seed: int) -> None:
    """All 64 scenes of one uneven batch; per-scene fields concatenated, with
    offsets ``<field>_off`` (length 65) for the variable-length ones."""
    import numpy as np

    torch, scenes, SBLConfig, fast_sbl = _import()
    batch = scenes.uneven_batch(batch_seed)
    out = {"grids": np.array([s.grid for s in batch], np.int64),
           "samples": np.array([s.y.shape for s in batch], np.int64),
           "y_sha256": np.array([y_digest(s.y) for s in batch]),
           "scene": np.array(f"uneven_batch({batch_seed})")}
    for profile in ("stable", "fast"):
        cfg = plan_config(SBLConfig, profile)
        per = [_solve_fields(fast_sbl(torch.from_numpy(s.y), s.grid, config=cfg), np) for s in batch]
        for k in per[0]:
            vals = [np.atleast_1d(p[k]) for p in per]
            out[f"{profile}_{k}"] = np.concatenate(vals)
            out[f"{profile}_{k}_off"] = np.concatenate([[0], np.cumsum([v.size for v in vals])]).astype(np.int64)
    np.savez_compressed(HERE / f"c4_b{batch_seed}.npz", **out)
    print("wrote", f"c4_b{batch_seed}")


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


JOBS = [("c3", "0"), ("c3", "1"), ("c3", "2"), ("c4", "0"), ("cg_c2", "0", "6")]


def main() -> None:
    if len(sys.argv) > 1:
        kind, args = sys.argv[1], [int(v) for v in sys.argv[2:]]
        {"c3": make_c3, "c4": make_c4, "cg_c2": make_cg_c2}[kind](*args)
        return
    reference_root()
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    for job in JOBS:
        subprocess.run([sys.executable, __file__, *job], check=True, env=env)


if __name__ == "__main__":
    main()
