"""Generate mode="cg" golden vectors by executing the reference FBME-SBL package.

Run in a container that holds the reference source tree (it does not
travel to GPU machines); give its root in FBME_REFERENCE_ROOT:

    FBME_REFERENCE_ROOT=<path to FBME-SBL> python tests/golden/make_golden_cg.py

For each case it runs the reference ``fast_sbl`` with ``mode="cg"`` and
``active_set=False`` on the CPU, once with complex128 input (the
reference's FP64 pipeline) and once with complex64 input (its FP32
pipeline), and stores the observations, the dense outputs of the FP64 run
(in single precision), the scalar outputs and per-iteration history of
both runs, and the reference's FP32-vs-FP64 gaps in ``tests/golden/cg/<case>.npz``.  The probes are
the reference's own CPU generator stream (``_make_probes`` with seed 0,
solver.py:5979-6000); tests regenerate them with the same call.  The FP32
vs FP64 gap of the reference itself is what the GPU parity tolerance is
measured against.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "cg"
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))
from make_golden_configs import reference_root  # noqa: E402

# (name, scene config, seeds stacked as a batch, max_iter)
CASES = [
    ("cg_c1_s0_it20", "c1", (0,), 20),
    ("cg_c1_s3_it24", "c1", (3,), 24),
    ("cg_c1_b2_it12", "c1", (1, 2), 12),
]


def _child(name: str, config: str, seeds: tuple[int, ...], max_iter: int) -> None:
    import numpy as np
    import torch

    sys.path.append(str(REPO / "fbme-sbl_b200"))
    sys.path.insert(0, reference_root())
    from fbme_b200 import scenes
    from torch_sbl.solver import SBLConfig, fast_sbl  # reference package

    torch.set_num_threads(8)
    scs = [scenes.config_scene(config, s) for s in seeds]
    y = np.stack([sc.y for sc in scs])
    grid = scs[0].grid
    out = {"y": y, "grid": np.array(grid), "seeds": np.array(seeds), "max_iter": np.array(max_iter),
           "x_true": np.stack([sc.x for sc in scs]).astype(np.complex64)}
    runs = {}
    for tag, dtype in (("f64", np.complex128), ("f32", np.complex64)):
        cfg = SBLConfig(mode="cg", active_set=False, max_iter=max_iter, device="cpu",
                        return_history=True)
        r = fast_sbl(torch.from_numpy(y.astype(dtype)), grid, config=cfg)
        runs[tag] = r
        if tag == "f64":  # dense fields of the FP64 run, stored in single precision
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
    # the reference's own FP32-vs-FP64 gap (relative L2 over the batch)
    def gap(a, b):
        a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
        return np.linalg.norm(a - b) / np.linalg.norm(b)
    out["gap_x"] = np.array(gap(runs["f32"].x.numpy(), runs["f64"].x.numpy()))
    out["gap_posterior_variance"] = np.array(gap(runs["f32"].posterior_variance.numpy(),
                                                 runs["f64"].posterior_variance.numpy()))
    out["gap_precision"] = np.array(gap(runs["f32"].precision.numpy(), runs["f64"].precision.numpy()))
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print("wrote", name)


def _probes() -> None:
    """Hadamard probes of the reference (solver.py:6001-6083) on a 32 x 24
    sample grid, to pin the host-side probe construction."""
    import numpy as np
    import torch

    sys.path.insert(0, reference_root())
    from torch_sbl.solver import _make_probes  # reference package

    out = {}
    for count in (8, 13, 32):
        z = _make_probes(2, 32 * 24, count, device=torch.device("cpu"), dtype=torch.float32, seed=5,
                         probe_type="hadamard", probe_shape=(32, 24))
        out[f"hadamard_{count}"] = z.numpy().astype(np.int8)
    z = _make_probes(2, 32 * 24, 8, device=torch.device("cpu"), dtype=torch.float32, seed=5)
    out["rademacher_8"] = z.numpy().astype(np.int8)
    OUT.mkdir(exist_ok=True)
    np.savez_compressed(OUT / "probes.npz", **out)
    print("wrote probes")


def main() -> None:
    if len(sys.argv) == 2 and sys.argv[1] == "probes":
        _probes()
        return
    if len(sys.argv) == 5:
        _child(sys.argv[1], sys.argv[2], tuple(int(v) for v in sys.argv[3].split(",")),
               int(sys.argv[4]))
        return
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    for name, config, seeds, max_iter in CASES:
        subprocess.run([sys.executable, __file__, name, config, ",".join(map(str, seeds)),
                        str(max_iter)], check=True, env=env)
    subprocess.run([sys.executable, __file__, "probes"], check=True, env=env)


if __name__ == "__main__":
    main()
