"""Learned warm start on the B200: what the trained network gains, the plain
fallback, and parity of the warm-started solve with the oracle.

Held-out scenes come from the learned-training distribution (256x256 grid,
128x128 prefix, K ~ U{100..400}, SNR ~ U[5, 25] dB) with seeds 2*10^6 ...,
which training never saw (training seeds are 10^6 ... 10^6 + 19999).
"""

import numpy as np
import pytest

from gpu_util import X_TOL, need_gpu, rel_l2

torch = pytest.importorskip("torch")

GRID, PREFIX = (256, 256), (128, 128)


def _batch(n, seed0=2_000_000):
    from fbme_b200 import scenes

    sc = [scenes.learned_scene(seed0 + i) for i in range(n)]
    y = np.stack([c.y for c in sc]).astype(np.complex64)
    x = np.stack([c.x.reshape(-1) for c in sc])
    return y, x


def _nmse(xh, x):
    xh = xh.reshape(x.shape[0], -1)
    return 10 * np.log10(np.sum(np.abs(xh - x) ** 2, 1) / np.sum(np.abs(x) ** 2, 1))


@pytest.mark.gpu
def test_trained_network_gains_over_plain_start():
    """At the warm plan's budget (1 UAMP sweep) the network's prior beats the
    backprojection start by > 0.1 dB, and the warm plan is at least as good
    as plain FBME-Stable with its own budget (within 0.1 dB)."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.learned import make_learned_plan, plain_config
    from torch_sbl_fastest_stable import make_stable_plan

    y, x = _batch(64)
    yt = torch.from_numpy(y).cuda()
    stable = make_stable_plan(yt, GRID, warmup=1)
    n_stable = _nmse(stable.replay(yt, synchronize=True).x.cpu().numpy(), x).mean()
    e1 = FBMEEngine(64, GRID, PREFIX, plain_config(1), torch.device("cuda", 0))
    e1.run(yt.view(64, -1))
    n_plain1 = _nmse(e1.result((64,)).x.cpu().numpy(), x).mean()
    learned = make_learned_plan(yt, GRID, warmup=1)
    n_learned = _nmse(learned.replay(yt, synchronize=True).x.cpu().numpy(), x).mean()
    print(f"NMSE dB: stable {n_stable:.3f}, plain 1 sweep {n_plain1:.3f}, learned 1 sweep {n_learned:.3f}, "
          f"fallbacks {learned.fallbacks}")
    assert n_learned < n_plain1 - 0.1
    assert n_learned < n_stable + 0.1
    assert learned.fallbacks < 16


@pytest.mark.gpu
def test_fallback_returns_the_plain_plan_result():
    need_gpu()
    from fbme_b200.learned import make_learned_plan
    from torch_sbl_fastest_stable import make_stable_plan

    y, _ = _batch(8, 2_100_000)
    yt = torch.from_numpy(y).cuda()
    learned = make_learned_plan(yt, GRID, warmup=1)
    learned.gamma_residual_max = -1.0  # every scene fails the check
    r = learned.replay(yt, synchronize=True)
    assert learned.fallbacks == 8
    p = make_stable_plan(yt, GRID, warmup=1).replay(yt, synchronize=True)
    assert torch.equal(r.x, p.x)
    assert torch.equal(r.posterior_variance, p.posterior_variance)
    assert torch.equal(r.negative_log_evidence, p.negative_log_evidence)


@pytest.mark.gpu
def test_one_forced_failure_is_resolved_on_the_device():
    """A single failed scene is re-solved by the plain plan inside the
    fallback graph; its rows become the plain result, every other row keeps
    the warm result."""
    need_gpu()
    from fbme_b200.learned import make_learned_plan
    from torch_sbl_fastest_stable import make_stable_plan

    y, _ = _batch(8, 2_150_000)
    yt = torch.from_numpy(y).cuda()
    learned = make_learned_plan(yt, GRID, warmup=1, fallback_capacity=4)
    warm = learned.replay(yt, synchronize=True, fallback=False)
    x_warm, nle_warm = warm.x.clone(), warm.negative_log_evidence.clone()
    passed_warm = learned.passed.clone()
    learned.force_fallback[5] = True
    r = learned.replay(yt)
    torch.cuda.current_stream().synchronize()  # stream order alone completes the results
    assert not bool(learned.passed[5]) and not bool(learned.overflow)
    p = make_stable_plan(yt, GRID, warmup=1).replay(yt, synchronize=True)
    assert torch.equal(r.x[5], p.x[5])
    assert torch.equal(r.posterior_variance[5], p.posterior_variance[5])
    assert torch.equal(r.negative_log_evidence[5], p.negative_log_evidence[5])
    keep = [i for i in range(8) if i != 5 and bool(passed_warm[i])]
    assert keep, "every warm scene failed its check"
    assert torch.equal(r.x[keep], x_warm[keep])
    assert torch.equal(r.negative_log_evidence[keep], nle_warm[keep])
    assert learned.fallbacks == 1 + int((~passed_warm).sum()) - int(not bool(passed_warm[5]))


@pytest.mark.gpu
def test_failures_beyond_the_capacity_are_resolved_on_synchronize():
    need_gpu()
    from fbme_b200.learned import make_learned_plan
    from torch_sbl_fastest_stable import make_stable_plan

    y, _ = _batch(8, 2_100_000)
    yt = torch.from_numpy(y).cuda()
    learned = make_learned_plan(yt, GRID, warmup=1, fallback_capacity=3)
    learned.force_fallback.fill_(True)
    learned.replay(yt)
    assert bool(learned.overflow)
    r = learned.replay(yt, synchronize=True)
    assert learned.fallbacks == 8
    p = make_stable_plan(yt, GRID, warmup=1).replay(yt, synchronize=True)
    assert torch.equal(r.x, p.x)
    assert torch.equal(r.noise_variance, p.noise_variance)


def _tensors(res):
    from dataclasses import fields

    return {f.name: getattr(res, f.name).clone() for f in fields(res)
            if isinstance(getattr(res, f.name), torch.Tensor)}


@pytest.mark.gpu
def test_pipelined_replays_equal_stream_ordered_replays():
    """Two warm plans take turns and each replay's fallback overlaps the next
    replay's warm solve; after synchronize() every replay's results equal
    the stream-ordered plan's."""
    need_gpu()
    from fbme_b200.learned import make_learned_plan

    ya, _ = _batch(8, 2_300_000)
    yb, _ = _batch(8, 2_300_100)
    ta, tb = torch.from_numpy(ya).cuda(), torch.from_numpy(yb).cuda()
    plain = make_learned_plan(ta, GRID, warmup=1)
    plain.force_fallback[[1, 6]] = True
    ra, rb = _tensors(plain.replay(ta, synchronize=True)), _tensors(plain.replay(tb, synchronize=True))
    pipe = make_learned_plan(ta, GRID, warmup=1, pipelined=True)
    pipe.force_fallback[[1, 6]] = True
    r1 = pipe.replay(ta)
    r2 = pipe.replay(tb)
    pipe.synchronize()
    assert r1 is not r2
    for ref, got in ((ra, r1), (rb, r2)):
        for k, v in ref.items():
            assert torch.equal(getattr(got, k), v), k


@pytest.mark.gpu
def test_warm_started_solve_matches_oracle_from_the_network_prior():
    """The warm plan is the plain algorithm started from the network's prior:
    the oracle restatement given the same prior agrees (x within 1e-4
    relative L2, identical support)."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.learned import DEFAULT_WEIGHTS, WarmStartNet, attach_warm_start, plain_config
    from oracle import fbme_oracle as O

    y, _ = _batch(2, 2_200_000)
    dev = torch.device("cuda", 0)
    yt = torch.from_numpy(y).cuda().view(2, -1)
    net = WarmStartNet.load(DEFAULT_WEIGHTS, dev)
    eng = FBMEEngine(2, GRID, PREFIX, plain_config(1), dev)
    ws = attach_warm_start(eng, net)
    eng.run(yt)
    x = eng.result((2,)).x.cpu().numpy().reshape(2, -1)
    bp = eng.state()["backprojection"].clone()
    out = net.predict(bp, *GRID).cpu().numpy().astype(np.float32)
    n = GRID[0] * GRID[1]
    dp = np.maximum(np.mean(np.abs(y.reshape(2, -1)) ** 2, axis=1), np.finfo(np.float32).eps).astype(np.float32)
    fl = np.maximum(dp * np.float32(1e-12), np.finfo(np.float32).tiny)
    prior0 = np.maximum((dp / np.float32(n))[:, None] * np.exp(np.clip(out, -40, 40)), fl[:, None])
    cfg = O.OracleConfig.stable(32)
    cfg.uamp_auto_iterations = False
    cfg.max_iter = 1
    cfg.uamp_min_iter = 1
    r = O.fast_sbl_uamp(y, GRID, cfg, initial_prior=prior0.astype(np.float32))
    xo = r["x"].reshape(2, -1)
    for b in range(2):
        assert set(np.flatnonzero(x[b])) == set(np.flatnonzero(xo[b]))
    assert rel_l2(x, xo) < X_TOL
    del ws


@pytest.mark.gpu
@pytest.mark.parametrize("grid,prefix", [(GRID, PREFIX), ((40, 48), (24, 32))])
def test_warm_prior_map_equals_the_attached_network(grid, prefix):
    """A caller-supplied log-prior map (here: the shipped network's output
    for A^H y, through the unfused layer kernels) warm-starts the plan
    exactly as the attached network (the fused network + prior kernel)
    does; the 40 x 48 grid has tiles cut by the image edge."""
    need_gpu()
    from fbme_b200.engine import FBMEEngine
    from fbme_b200.learned import (DEFAULT_WEIGHTS, WarmStartNet, attach_warm_prior_map, attach_warm_start,
                                   plain_config)

    if grid == GRID:
        y, _ = _batch(4, 2_400_000)
    else:
        rng = np.random.default_rng(11)
        m = prefix[0] * prefix[1]
        y = (rng.normal(size=(4, m)) + 1j * rng.normal(size=(4, m))).astype(np.complex64)
    dev = torch.device("cuda", 0)
    yt = torch.from_numpy(y).cuda().view(4, -1)
    net = WarmStartNet.load(DEFAULT_WEIGHTS, dev)
    a = FBMEEngine(4, grid, prefix, plain_config(1), dev)
    ws = attach_warm_start(a, net)
    a.run(yt)
    b = FBMEEngine(4, grid, prefix, plain_config(1), dev)
    prior_map = net.predict(b.dft_adjoint(yt), *grid).contiguous()
    attach_warm_prior_map(b, prior_map)
    b.run(yt)
    torch.cuda.synchronize()
    for f in ("x", "posterior_variance", "negative_log_evidence", "noise_variance"):
        assert torch.equal(a.out[f], b.out[f]), f
    attach_warm_prior_map(b, None)  # back to the plain initialisation
    b.run(yt)
    c = FBMEEngine(4, grid, prefix, plain_config(1), dev)
    c.run(yt)
    torch.cuda.synchronize()
    assert torch.equal(b.out["x"], c.out["x"])
    del ws
