"""The oracle's global certificate and support repairs (certified_hybrid_uamp,
torch_sbl/solver.py:300-316, 3522-3588, 3219-3317, 4511-4628, 5388-5460)
against fixtures produced by the reference itself
(tests/golden/make_golden_configs.py make_certified)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from golden_util import CERT_FILES, certificate_checks, plan_case
from oracle import fbme_oracle as O


def test_fixtures_present():
    assert len(CERT_FILES) >= 4


@pytest.mark.parametrize("path", CERT_FILES, ids=[Path(p).stem for p in CERT_FILES])
def test_oracle_matches_reference_certificate(path):
    y, grid, g = plan_case(path)
    over = dict(uamp_polish_support_repairs=int(g["repairs"]))
    if float(g["fwer"]) > 0:
        over["uamp_polish_familywise_error_rate"] = float(g["fwer"])
    o = O.fast_sbl_uamp(y, grid, O.OracleConfig.certified_hybrid_uamp(**over))
    res = {k: v for k, v in o.items()}
    res.update(x=o["x"].reshape(-1), pv=o["posterior_variance"].reshape(-1),
               precision=o["precision"].reshape(-1))
    certificate_checks(res, g, x_rtol=1e-5, pv_rtol=1e-4, cert_rtol=1e-5, tag=Path(path).stem)


def test_ratio_threshold_inverts_the_gain():
    for tol in (1e-6, 1e-3, 0.5):
        rho = O.ratio_threshold_for_evidence_tolerance(tol)
        assert rho > 1.0 and abs((rho - 1.0 - np.log(rho)) - tol) <= 1e-12 + 1e-9 * tol
    assert O.ratio_threshold_for_evidence_tolerance(0.0) == 1.0
