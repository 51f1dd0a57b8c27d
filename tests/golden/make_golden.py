"""Generate golden vectors by executing the reference FBME-SBL package.

Run in a container that holds the reference source tree (it does not
travel to GPU machines); give its root in FBME_REFERENCE_ROOT:

    FBME_REFERENCE_ROOT=<path to FBME-SBL> python tests/golden/make_golden.py

For each seeded synthetic scene it runs the reference ``fast_sbl`` with the
exact FBME-Stable / FBME-Fast plan configurations on the CPU
(``uamp_backend="torch"``, the reference's own CPU arithmetic path,
torch_sbl/solver.py:2808-2850) and stores the input observation and the
result fields in a compressed ``.npz``.  Outputs that are zero / floor
outside the final active set are stored sparsely (active indices plus
values) to keep the fixtures small.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))
from make_golden_configs import reference_root  # noqa: E402

CASES = [
    # (name, config, seed, profiles)
    ("c1_s0", "c1", 0), ("c1_s1", "c1", 1), ("c1_s2", "c1", 2),
    ("c2_s0", "c2", 0), ("c2_s1", "c2", 1),
    ("rtx_s200", "rtx", 200),
]


def _child(name: str, config: str, seed: int) -> None:
    import numpy as np
    import torch

    sys.path.insert(0, reference_root())
    sys.path.append(str(REPO / "fbme-sbl_b200"))
    from fbme_b200 import scenes
    from torch_sbl.solver import SBLConfig, fast_sbl  # reference package

    torch.set_num_threads(4)
    if config == "rtx":
        sc = scenes.point_scene((40, 32), (20, 16), 21, 10.0, seed, "cn")
    else:
        sc = scenes.config_scene(config, seed)
    y = torch.from_numpy(sc.y)
    out = {"y": sc.y, "grid": np.array(sc.grid), "x_true": sc.x.astype(np.complex64)}
    for profile in ("stable", "fast"):
        over = dict(device="cpu", uamp_backend="torch", uamp_polish_size=32,
                    uamp_polish_compute_truncation_diagnostic=False)
        if profile == "stable":
            over.update(uamp_polish_iterations=3, uamp_polish_residual_exchange_size=12,
                        uamp_polish_fixed_budget_diagnostics=True)
        else:
            over.update(uamp_polish_iterations=2, uamp_polish_residual_exchange_size=0,
                        uamp_polish_fixed_budget_diagnostics=False)
        cfg = SBLConfig.paper_hybrid_uamp(**over)
        r = fast_sbl(y, sc.grid, config=cfg)
        x = r.x.numpy().reshape(-1)
        act = np.flatnonzero(x != 0)
        pv = r.posterior_variance.numpy().reshape(-1)
        prec = r.precision.numpy().reshape(-1)
        mask = r.support_mask.numpy().reshape(-1)
        p = profile + "_"
        out[p + "active"] = act.astype(np.int64)
        out[p + "x_active"] = x[act]
        out[p + "pv_active"] = pv[act]
        out[p + "precision_active"] = prec[act]
        inactive = np.ones(x.size, bool)
        inactive[act] = False
        out[p + "pv_inactive_unique"] = np.unique(pv[inactive])
        out[p + "precision_inactive_unique"] = np.unique(prec[inactive])
        out[p + "mask_indices"] = np.flatnonzero(mask).astype(np.int64)
        for f in ("noise_variance", "effective_dof", "negative_log_evidence",
                  "evidence_trace", "support_score_threshold",
                  "fixed_budget_gamma_residual", "fixed_budget_noise_residual",
                  "fixed_budget_objective_decrease", "fixed_budget_monotone",
                  "support_exchanges_accepted"):
            v = getattr(r, f)
            if v is not None:
                out[p + f] = v.numpy()
        out[p + "iterations"] = np.array(r.iterations)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print("wrote", name)


def main() -> None:
    if len(sys.argv) == 4 and sys.argv[1] != "--all":
        _child(sys.argv[1], sys.argv[2], int(sys.argv[3]))
        return
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    for name, config, seed in CASES:
        subprocess.run([sys.executable, __file__, name, config, str(seed)], check=True, env=env)


if __name__ == "__main__":
    main()
