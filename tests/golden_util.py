"""Loading of the reference-generated golden fixtures (tests/golden).

Fixtures made by make_golden.py store the observation ``y``.  Those made by
make_golden_configs.py store the generator call and the SHA-256 of its
observation instead; the observation is regenerated here with the committed
scene generator and checked against the digest, so a changed generator
fails loudly rather than comparing against the wrong scene.
"""

from __future__ import annotations

import glob
import hashlib
import re
from pathlib import Path

import numpy as np

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"

# single-scene plan fixtures (one scene, both profiles)
PLAN_FILES = sorted(p for p in glob.glob(str(GOLDEN_DIR / "*.npz"))
                    if not Path(p).name.startswith(("c4_", "masked_", "cert_")))
# single-scene fixtures solved under an observation mask (key "mask")
MASKED_FILES = sorted(glob.glob(str(GOLDEN_DIR / "masked_*.npz")))
# single-scene fixtures solved under certified_hybrid_uamp (global
# certificate and support repairs; keys "repairs", "fwer")
CERT_FILES = sorted(glob.glob(str(GOLDEN_DIR / "cert_*.npz")))
# batched-uneven fixtures (64 scenes each)
UNEVEN_FILES = sorted(glob.glob(str(GOLDEN_DIR / "c4_*.npz")))


def _digest(y) -> str:
    return hashlib.sha256(np.ascontiguousarray(y, dtype=np.complex64).tobytes()).hexdigest()


def plan_case(path):
    """(y [M1, M2] complex64, grid, fixture) of a single-scene fixture."""
    g = np.load(path)
    grid = tuple(int(v) for v in g["grid"])
    if "y" in g.files:
        return g["y"], grid, g
    from fbme_b200 import scenes

    m = re.fullmatch(r"config_scene\('(\w+)', (\d+)\)", str(g["scene"]))
    assert m, str(g["scene"])
    y = scenes.config_scene(m.group(1), int(m.group(2))).y
    assert _digest(y) == str(g["y_sha256"]), "scene generator changed: fixture no longer matches"
    return y, grid, g


def uneven_case(path):
    """(list of scenes, fixture) of a batched-uneven fixture."""
    from fbme_b200 import scenes

    g = np.load(path)
    m = re.fullmatch(r"uneven_batch\((\d+)\)", str(g["scene"]))
    assert m, str(g["scene"])
    batch = scenes.uneven_batch(int(m.group(1)))
    assert [_digest(s.y) for s in batch] == [str(v) for v in g["y_sha256"]], "scene generator changed"
    return batch, g


def scene_field(g, key: str, i: int):
    """Field ``key`` of scene i of a packed batched fixture."""
    off = g[key + "_off"]
    return g[key].reshape(-1)[off[i]:off[i + 1]]


def scene_fields(g, profile: str, i: int) -> dict:
    """Every field of scene i under ``profile`` as a single-scene fixture has them."""
    p = profile + "_"
    out = {}
    for k in g.files:
        if k.startswith(p) and not k.endswith("_off"):
            v = scene_field(g, k, i)
            out[k] = v if k[len(p):] in ("active", "x_active", "pv_active", "precision_active",
                                         "pv_inactive_unique", "precision_inactive_unique",
                                         "mask_indices", "evidence_trace") else v.reshape(())
    return out


# Parity bar on ill-conditioned scenes (C3 and a few C4 scenes): x within
# SENS_FACTOR times the reference's own sensitivity (the largest change of
# its FP32 result under input perturbations the size of the split-BF16 DFT
# rounding, make_golden_configs.PERTURBATION), when that exceeds the fixed
# bar.  Measured: the device lands within 1.8x of it on every C3 scene.
SENS_FACTOR = 4.0


def sensitivity(g, profile: str, i: int | None = None) -> tuple[float, float]:
    """(x, posterior variance) sensitivity of a fixture scene, 0 if absent."""
    if "sens_" + profile + "_x" not in g.files:
        return 0.0, 0.0
    sx, sv = g["sens_" + profile + "_x"], g["sens_" + profile + "_pv"]
    if i is not None:
        sx, sv = sx[i], sv[i]
    return float(sx), float(sv)


def certificate_checks(res, g, *, x_rtol: float, pv_rtol: float, cert_rtol: float, tag: str = "") -> None:
    """Compare a certified solve (dict-like ``res`` of numpy arrays: x, pv,
    precision flattened, certificate fields) with a ``cert_*`` fixture.

    The bars: identical support, x within ``x_rtol`` relative L2, posterior
    variance within ``pv_rtol`` on the support, the inactive certificate
    (ratio, gain, variance) within ``cert_rtol``, indices, counts and flags
    equal.  The active gains are differences of O(|deletion delta|) FP32
    values (solver.py:3277-3290: current_delta - optimal_delta), so they
    carry an absolute error of a few ulp of max|deletion delta|: they are
    compared at 16 such ulp, and the best active atom (with its optimal
    variance) only when its gain stands clear of that noise.
    """
    x, pv, prec = res["x"], res["pv"], res["precision"]
    act = np.flatnonzero(x != 0)
    assert np.array_equal(act, g["active"]), f"{tag}: support differs"
    xr = g["x_active"]
    assert np.linalg.norm(x[act] - xr) / np.linalg.norm(xr) <= x_rtol, tag
    assert np.max(np.abs(pv[act] - g["pv_active"]) / g["pv_active"]) <= pv_rtol, tag
    assert np.allclose(prec[act], g["precision_active"], rtol=pv_rtol), tag
    for f in ("inactive_max_evidence_ratio", "inactive_evidence_gain", "inactive_optimal_variance",
              "inactive_penalized_evidence_gain", "negative_log_evidence", "noise_variance"):
        assert np.allclose(res[f], g[f], rtol=cert_rtol, atol=0), (tag, f, res[f], g[f])
    tr = np.asarray(res["evidence_trace"]).reshape(-1)
    assert tr.shape == g["evidence_trace"].reshape(-1).shape, tag
    assert np.allclose(tr, g["evidence_trace"].reshape(-1), rtol=cert_rtol), (tag, tr)
    for f in ("inactive_best_index", "support_repairs_accepted", "support_exchanges_accepted",
              "coordinate_stationary", "type2_coordinate_stationary", "type2_map_coordinate_stationary"):
        assert int(np.asarray(res[f]).reshape(())) == int(g[f].reshape(())), (tag, f, res[f], g[f])
    for f in ("inactive_ratio_threshold", "stationarity_ratio_threshold"):
        assert np.float32(np.asarray(res[f]).reshape(())) == np.float32(g[f].reshape(())), (tag, f)
    if "familywise_ratio_threshold" in g.files:
        assert np.float32(np.asarray(res["familywise_ratio_threshold"]).reshape(())) == np.float32(
            g["familywise_ratio_threshold"].reshape(())), tag
        for f in ("familywise_no_discovery", "familywise_support_certified"):
            assert bool(np.asarray(res[f]).reshape(())) == bool(g[f].reshape(())), (tag, f)
    else:
        assert res.get("familywise_no_discovery") is None, tag
    ulp = float(np.spacing(np.float32(abs(float(g["active_max_deletion_gain"])))))
    atol = 16.0 * ulp
    for f in ("active_max_evidence_gain", "active_penalized_evidence_gain", "active_max_deletion_gain"):
        assert abs(float(res[f]) - float(g[f])) <= atol + 1e-5 * abs(float(g[f])), (tag, f, res[f], g[f])
    if float(g["active_max_evidence_gain"]) > 2.0 * atol:
        assert int(res["active_best_index"]) == int(g["active_best_index"]), tag
        assert np.isclose(float(res["active_optimal_variance"]), float(g["active_optimal_variance"]),
                          rtol=max(cert_rtol, 1e-3)), tag
    assert int(res["active_best_index"]) in set(int(v) for v in act), tag
