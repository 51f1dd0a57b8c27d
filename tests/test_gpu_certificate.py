"""Global certificate and support repairs (certified_hybrid_uamp) on the B200
against the reference and the oracle.

The fixtures (tests/golden/cert_*.npz, make_golden_configs.py
make_certified) are the reference's sbl_2d under certified_hybrid_uamp at
64^2/32^2 and 256^2/128^2, with 1-3 support repairs (kept: 0, 1, 1, 2) and
one familywise threshold.  Bar: identical support, x within 1e-4 relative L2,
posterior variance within 1e-3, the inactive certificate and the evidence
within 1e-4, indices, counts and flags equal; the active gains at 16 ulp of
the largest deletion delta (golden_util.certificate_checks).
"""

from pathlib import Path

import numpy as np
import pytest

from golden_util import CERT_FILES, certificate_checks, plan_case
from gpu_util import need_gpu

torch = pytest.importorskip("torch")

FIELDS = ("inactive_max_evidence_ratio", "inactive_best_index", "inactive_evidence_gain",
          "inactive_optimal_variance", "support_repairs_accepted", "support_exchanges_accepted",
          "active_max_evidence_gain", "active_best_index", "active_optimal_variance", "active_max_deletion_gain",
          "coordinate_stationary", "inactive_ratio_threshold", "type2_coordinate_stationary",
          "stationarity_ratio_threshold", "familywise_ratio_threshold", "familywise_no_discovery",
          "familywise_support_certified", "inactive_penalized_evidence_gain", "active_penalized_evidence_gain",
          "type2_map_coordinate_stationary", "noise_variance", "effective_dof", "negative_log_evidence",
          "evidence_trace")


def _overrides(repairs: int, fwer: float) -> dict:
    over = dict(uamp_polish_support_repairs=repairs)
    if fwer > 0:
        over["uamp_polish_familywise_error_rate"] = fwer
    return over


def _numpy_fields(r, b=None) -> dict:
    pick = (lambda t: t) if b is None else (lambda t: t[b])
    out = {}
    for f in FIELDS:
        v = getattr(r, f)
        out[f] = None if v is None else pick(v).detach().cpu().numpy()
    out.update(x=pick(r.x).reshape(-1).cpu().numpy(), pv=pick(r.posterior_variance).reshape(-1).cpu().numpy(),
               precision=pick(r.precision).reshape(-1).cpu().numpy())
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("path", CERT_FILES, ids=lambda p: Path(p).stem)
def test_certified_sbl_2d_matches_reference(path):
    need_gpu()
    from fbme_b200.config import SBLConfig
    from torch_sbl import sbl_2d

    y_np, grid, g = plan_case(path)
    cfg = SBLConfig.certified_hybrid_uamp(device="cuda", **_overrides(int(g["repairs"]), float(g["fwer"])))
    r = sbl_2d(torch.from_numpy(y_np).cuda(), grid, config=cfg)
    assert int(r.status) == 0
    assert r.evidence_trace.shape == (1, cfg.uamp_polish_iterations + int(g["repairs"]))
    certificate_checks(_numpy_fields(r), g, x_rtol=1e-4, pv_rtol=1e-3, cert_rtol=1e-4, tag=Path(path).stem)


@pytest.mark.gpu
def test_certified_batch_matches_oracle():
    """Eight 64^2/32^2 scenes in one call, three repairs and the familywise
    threshold, each scene against the oracle's certified solve."""
    need_gpu()
    from fbme_b200 import scenes
    from fbme_b200.config import SBLConfig
    from oracle import fbme_oracle as O
    from torch_sbl import sbl_2d

    over = _overrides(3, 0.05)
    ys = np.stack([scenes.config_scene("c1", 40 + i).y for i in range(8)])
    grid = scenes.config_scene("c1", 40).grid
    r = sbl_2d(torch.from_numpy(ys).cuda(), grid, config=SBLConfig.certified_hybrid_uamp(device="cuda", **over))
    o = O.fast_sbl_uamp(ys, grid, O.OracleConfig.certified_hybrid_uamp(**over))
    kept = 0
    for b in range(ys.shape[0]):
        ref = {k: (v[b] if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == ys.shape[0] else v)
               for k, v in o.items()}
        g = dict(ref)
        x = ref["x"].reshape(-1)
        act = np.flatnonzero(x != 0)
        g.update(active=act, x_active=x[act], pv_active=ref["posterior_variance"].reshape(-1)[act],
                 precision_active=ref["precision"].reshape(-1)[act])
        g = {k: np.asarray(v) for k, v in g.items() if v is not None}

        class _G(dict):
            files = property(lambda self: list(self.keys()))

        certificate_checks(_numpy_fields(r, b), _G(g), x_rtol=1e-4, pv_rtol=1e-3, cert_rtol=1e-4, tag=f"scene {b}")
        kept += int(r.support_repairs_accepted[b])
    assert int(r.status.abs().sum()) == 0
    assert kept > 0  # the repair path is exercised


@pytest.mark.gpu
def test_certificate_off_leaves_outputs_unchanged():
    """global certificate with zero repairs changes no reconstruction field."""
    need_gpu()
    from fbme_b200 import scenes
    from fbme_b200.config import SBLConfig
    from torch_sbl import sbl_2d

    sc = scenes.config_scene("c2", 3)
    y = torch.from_numpy(sc.y).cuda()
    base = SBLConfig.fast_hybrid_uamp(device="cuda", uamp_polish_iterations=4)
    r0 = sbl_2d(y, sc.grid, config=base)
    r1 = sbl_2d(y, sc.grid, config=SBLConfig.certified_hybrid_uamp(device="cuda", uamp_polish_support_repairs=0))
    assert torch.equal(r0.x, r1.x) and torch.equal(r0.posterior_variance, r1.posterior_variance)
    assert torch.equal(r0.evidence_trace, r1.evidence_trace)
    assert r0.inactive_max_evidence_ratio is None and r1.inactive_max_evidence_ratio is not None


def test_host_ratio_threshold_matches_reference():
    from fbme_b200.engine import ratio_threshold_for_evidence_tolerance

    _, _, g = plan_case(CERT_FILES[0])
    assert np.float32(ratio_threshold_for_evidence_tolerance(1e-6)) == np.float32(g["stationarity_ratio_threshold"])


def test_unbuilt_research_options_are_refused():
    from fbme_b200.config import SBLConfig
    from fbme_b200.engine import check_supported

    with pytest.raises(NotImplementedError, match="uamp_polish_support_growth_steps"):
        check_supported(SBLConfig.taes_hybrid_uamp(uamp_backend="torch"))
    check_supported(SBLConfig.certified_hybrid_uamp())
    with pytest.raises(NotImplementedError, match="at most 8"):
        check_supported(SBLConfig.certified_hybrid_uamp(uamp_polish_iterations=6, uamp_polish_support_repairs=3))
