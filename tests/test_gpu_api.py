"""Drop-in API behaviour on the GPU: plan validation errors, eager sbl_2d,
host-side fault injection reported through the per-scene status word."""

import numpy as np
import pytest

from gpu_util import need_gpu, rel_l2

torch = pytest.importorskip("torch")


@pytest.mark.gpu
def test_replay_input_validation():
    need_gpu()
    from fbme_b200 import scenes
    from torch_sbl_fastest_stable import make_stable_plan

    s = scenes.config_scene("c1", 0)
    y = torch.from_numpy(s.y).cuda()
    plan = make_stable_plan(y, (64, 64), warmup=1)
    with pytest.raises(ValueError):
        plan.replay(y.cpu())
    with pytest.raises(ValueError):
        plan.replay(y.to(torch.complex128))
    with pytest.raises(ValueError):
        plan.replay(y[:16])
    with pytest.raises(ValueError):
        make_stable_plan(y.to(torch.complex128), (64, 64))
    with pytest.raises(ValueError):
        make_stable_plan(y.cpu(), (64, 64))


@pytest.mark.gpu
def test_eager_sbl_2d_uamp_preset_matches_plan():
    need_gpu()
    from fbme_b200 import scenes
    from torch_sbl import SBLConfig, sbl_2d
    from torch_sbl_fastest_stable import make_stable_plan

    s = scenes.config_scene("c1", 2)
    y = torch.from_numpy(s.y).cuda()
    cfg = SBLConfig.realtime_hybrid_uamp(uamp_polish_size=32)
    eager = sbl_2d(y, (64, 64), config=cfg)
    plan = make_stable_plan(y, (64, 64), warmup=1).replay(y, synchronize=True)
    assert torch.equal(eager.x, plan.x)
    assert eager.x.data_ptr() != plan.x.data_ptr()


@pytest.mark.gpu
def test_fast_hybrid_preset_matches_oracle():
    """SBLConfig.fast_hybrid_uamp (adaptive damping, offset 1) through sbl_2d."""
    need_gpu()
    from fbme_b200 import scenes
    from oracle import fbme_oracle as O
    from torch_sbl import SBLConfig, sbl_2d

    s = scenes.config_scene("c2", 5)
    y = torch.from_numpy(s.y).cuda()
    res = sbl_2d(y, (256, 256), config=SBLConfig.fast_hybrid_uamp(device="cuda"))
    ref = O.fast_sbl_uamp(s.y, (256, 256), O.OracleConfig.fast_hybrid_uamp())
    x, xr = res.x.cpu().numpy(), ref["x"]
    assert set(np.flatnonzero(x)) == set(np.flatnonzero(xr))
    assert rel_l2(x, xr) < 1e-4


@pytest.mark.gpu
def test_nonfinite_input_sets_status_without_fault():
    """Fault injection on the host: NaN observations must surface as the
    NONFINITE status bit, and the context must stay usable."""
    need_gpu()
    from fbme_b200 import _native as nat
    from fbme_b200 import scenes
    from torch_sbl_fastest_stable import make_stable_plan

    good = [scenes.config_scene("c1", i).y for i in range(3)]
    y = torch.from_numpy(np.stack(good)).cuda()
    plan = make_stable_plan(y, (64, 64), warmup=1)
    bad = y.clone()
    bad[1, 3, 4] = complex(float("nan"), 0.0)
    r = plan.replay(bad, synchronize=True)
    st = r.status.cpu().numpy()
    assert st[1] & nat.STATUS_NONFINITE
    assert st[0] == 0 and st[2] == 0
    r = plan.replay(y, synchronize=True)
    assert int(r.status.abs().sum()) == 0


@pytest.mark.gpu
def test_unbuilt_modes_raise():
    need_gpu()
    from torch_sbl import SBLConfig, sbl_2d

    # dense mode is built up to 4096 samples
    y = torch.zeros(128, 64, dtype=torch.complex64, device="cuda")
    with pytest.raises(NotImplementedError):
        sbl_2d(y, (256, 256), config=SBLConfig(mode="dense", device="cuda"))
