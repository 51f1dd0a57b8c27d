"""Host pipeline (fbme_b200.streaming) on the B200: batches from pinned
host memory, copies overlapped with solves, must give exactly the plan's
own results, batch by batch, in compact and dense form."""

import numpy as np
import pytest

from gpu_util import need_gpu

torch = pytest.importorskip("torch")


@pytest.mark.gpu
@pytest.mark.parametrize("dense", [False, True])
def test_pipeline_results_equal_direct_replays(dense):
    need_gpu()
    from fbme_b200 import scenes
    from fbme_b200.streaming import HostPipeline
    from torch_sbl_fastest_stable import make_stable_plan

    grid, B, steps = (64, 64), 4, 5
    batches = [np.stack([scenes.config_scene("c1", 100 * j + i).y for i in range(B)]) for j in range(steps)]
    y0 = torch.from_numpy(batches[0]).cuda()
    plan = make_stable_plan(y0, grid, warmup=1)
    expect = []
    for yb in batches:
        r = plan.replay(torch.from_numpy(yb).cuda(), synchronize=True)
        expect.append((r.x.cpu().clone(), r.noise_variance.cpu().clone()))
    pipe = HostPipeline(plan, dense=dense)
    hosts = [torch.from_numpy(yb).pin_memory() for yb in batches]
    outs = [pipe.host_result() for _ in range(steps)]
    for yh, out in zip(hosts, outs):
        pipe.submit(yh, out)
    pipe.synchronize()
    for (x, nv), out in zip(expect, outs):
        assert torch.equal(out.dense_x(grid), x)
        assert torch.equal(out.noise_variance, nv)
        assert int(out.status.abs().sum()) == 0
        if not dense:
            # the compact form is the active set: K distinct indices
            assert out.active_indices.shape == (B, 32)
            assert all(len(set(row.tolist())) == 32 for row in out.active_indices)


@pytest.mark.gpu
def test_pipeline_rejects_a_wrong_shape():
    need_gpu()
    from fbme_b200 import scenes
    from fbme_b200.streaming import HostPipeline
    from torch_sbl_fastest_stable import make_fastest_plan

    y = torch.from_numpy(np.stack([scenes.config_scene("c1", i).y for i in range(2)])).cuda()
    pipe = HostPipeline(make_fastest_plan(y, (64, 64), warmup=1))
    with pytest.raises(ValueError):
        pipe.submit(torch.zeros(3, 32, 32, dtype=torch.complex64).pin_memory(), pipe.host_result())
