"""Observation masks (non-rectangular sampling) on the B200 against the
reference.

The fixtures (tests/golden/masked_*.npz, make_golden_configs.py) are the
reference's sbl_2d with an observation_mask under the FBME-Stable / Fast
configurations: a seeded random mask keeping ~70 % of the samples, and an
elliptical aperture inscribed in the M1 x M2 block, at 64^2/32^2 and
256^2/128^2.  Both the masked plans and masked sbl_2d must meet the parity
bar: identical support, x within 1e-4 relative L2 (or SENS_FACTOR times the
reference's own sensitivity where that is larger), posterior variance within
1e-3, scalars within 1e-4, the sweep budget of the observed count.
"""

from pathlib import Path

import numpy as np
import pytest

from golden_util import MASKED_FILES, plan_case, sensitivity
from gpu_util import need_gpu

torch = pytest.importorskip("torch")


def _check(res, g, profile, label):
    from test_gpu_parity import _check_plan_fields

    _check_plan_fields(res, g, profile, sensitivity(g, profile), label=label)


@pytest.mark.gpu
@pytest.mark.parametrize("profile", ["stable", "fast"])
@pytest.mark.parametrize("path", MASKED_FILES, ids=lambda p: Path(p).stem)
def test_masked_plan_matches_reference(path, profile):
    need_gpu()
    from torch_sbl_fastest_stable import make_fastest_plan, make_stable_plan

    y_np, grid, g = plan_case(path)
    mask = torch.from_numpy(g["mask"]).cuda()
    y = torch.from_numpy(y_np).cuda()
    make = make_stable_plan if profile == "stable" else make_fastest_plan
    plan = make(y, grid, warmup=1, observation_mask=mask)
    res = plan.replay(y, synchronize=True)
    _check(res, g, profile, f"{Path(path).stem} plan")
    # unobserved samples are ignored: changing them changes nothing
    y2 = y.clone()
    y2[~mask] = 1e3 + 1e3j
    r2 = plan.replay(y2, synchronize=True)
    assert torch.equal(r2.x, res.x)


@pytest.mark.gpu
@pytest.mark.parametrize("path", MASKED_FILES[:2], ids=lambda p: Path(p).stem)
def test_masked_sbl_2d_matches_reference(path):
    need_gpu()
    from fbme_b200.config import fbme_profile_config
    from torch_sbl import sbl_2d

    y_np, grid, g = plan_case(path)
    y = torch.from_numpy(y_np).cuda()
    res = sbl_2d(y, grid, config=fbme_profile_config("stable"), observation_mask=torch.from_numpy(g["mask"]))
    assert res.mode == "uamp"
    _check(res, g, "stable", f"{Path(path).stem} sbl_2d")


@pytest.mark.gpu
def test_full_mask_equals_the_unmasked_plan():
    """A mask that keeps every sample takes the masked code path (2-D Gram
    table, masked messages) and must give the unmasked plan's result to
    rounding: the 2-D table equals the product of the Dirichlet kernels."""
    need_gpu()
    from fbme_b200 import scenes
    from gpu_util import rel_l2
    from torch_sbl_fastest_stable import make_stable_plan

    sc = scenes.config_scene("c1", 3)
    y = torch.from_numpy(sc.y).cuda()
    full = torch.ones(sc.y.shape, dtype=torch.bool, device="cuda")
    a = make_stable_plan(y, sc.grid, warmup=1).replay(y, synchronize=True)
    b = make_stable_plan(y, sc.grid, warmup=1, observation_mask=full).replay(y, synchronize=True)
    xa, xb = a.x.cpu().numpy(), b.x.cpu().numpy()
    assert set(np.flatnonzero(xa)) == set(np.flatnonzero(xb))
    assert rel_l2(xb, xa) < 1e-5
    assert b.iterations == a.iterations


@pytest.mark.gpu
def test_mask_contract_errors():
    need_gpu()
    from fbme_b200 import scenes
    from fbme_b200.config import fbme_profile_config
    from torch_sbl import sbl_2d
    from torch_sbl_fastest_stable import make_stable_plan

    sc = scenes.config_scene("c1", 0)
    y = torch.from_numpy(sc.y).cuda()
    with pytest.raises(ValueError, match="at least one sample"):
        sbl_2d(y, sc.grid, config=fbme_profile_config("stable"),
               observation_mask=torch.zeros(sc.y.shape, dtype=torch.bool))
    with pytest.raises(ValueError, match="trailing data dimensions"):
        sbl_2d(y, sc.grid, config=fbme_profile_config("stable"), observation_mask=torch.ones(4, 4, dtype=torch.bool))
    with pytest.raises(ValueError, match="observation_mask must have shape"):
        make_stable_plan(y, sc.grid, warmup=1, observation_mask=torch.ones(3, 3, dtype=torch.bool))
