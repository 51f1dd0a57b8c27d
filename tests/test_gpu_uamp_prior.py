"""The unfused variational ARD prior update (fbme_uamp_prior_update, the
reference's uamp_prior_update at torch_sbl/triton_kernels.py:670-735)
against a plain PyTorch float32 evaluation of the same expression, one
operation at a time: bit-exact.  Covers the 16-byte path, ragged rows (n
not a multiple of 4), a misaligned view, and both clamps."""

import numpy as np
import pytest

from gpu_util import need_gpu

torch = pytest.importorskip("torch")


def _torch_reference(mean, pv, old, floor, hyper_shape, hyper_rate, damping, maximum):
    f = lambda v: torch.tensor(v, dtype=torch.float32, device=mean.device)  # noqa: E731
    m2 = (mean.real * mean.real + mean.imag * mean.imag) + pv
    cand = (m2 + f(hyper_rate)) / (f(1.0) + f(hyper_shape))
    cand = torch.maximum(floor[:, None], torch.minimum(f(maximum), cand))
    upd = f(damping) * old + (f(1.0) - f(damping)) * cand
    return torch.maximum(upd, floor[:, None])


def _inputs(batch, n, seed, offset=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    mean = torch.complex(torch.randn(batch, n + offset, generator=g), torch.randn(batch, n + offset, generator=g))
    pv = torch.rand(batch, n + offset, generator=g) * 0.1
    old = torch.rand(batch, n + offset, generator=g) * 2.0
    floor = torch.rand(batch, generator=g) * 0.05
    mean[:, :7] *= 1e-4  # below the floor
    mean[:, 7:11] *= 1e3  # above the maximum
    t = [v.cuda() for v in (mean, pv, old)]
    if offset:
        t = [v.reshape(-1)[offset: offset + batch * n].reshape(batch, n) for v in t]
    return (*t, floor.cuda())


@pytest.mark.gpu
@pytest.mark.parametrize("batch,n,offset", [(3, 4096, 0), (2, 1001, 0), (2, 512, 1)])
@pytest.mark.parametrize("damping", [0.15, 0.0])
def test_prior_update_matches_float32_reference_bitwise(batch, n, offset, damping):
    need_gpu()
    from fbme_b200.engine import uamp_prior_update

    mean, pv, old, floor = _inputs(batch, n, 7 + n, offset)
    kw = dict(hyper_shape=1e-8, hyper_rate=1e-8, damping=damping, maximum=50.0)
    got = uamp_prior_update(mean.contiguous(), pv.contiguous(), old.contiguous(), floor, **kw) if offset \
        else uamp_prior_update(mean, pv, old, floor, **kw)
    ref = _torch_reference(mean, pv, old, floor, **kw)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    assert bool((got >= floor[:, None]).all())
    # the rounding-free value agrees to float32 resolution
    m64 = mean.to(torch.complex128)
    cand = torch.maximum(((m64.abs() ** 2 + pv.double() + 1e-8) / (1 + 1e-8)).clamp(max=50.0),
                         floor.double()[:, None])
    exact = torch.maximum(damping * old.double() + (1 - damping) * cand, floor.double()[:, None])
    np.testing.assert_allclose(got.double().cpu().numpy(), exact.cpu().numpy(), rtol=3e-7)


@pytest.mark.gpu
def test_prior_update_contract_errors():
    need_gpu()
    from fbme_b200.engine import uamp_prior_update

    mean, pv, old, floor = _inputs(2, 64, 1)
    kw = dict(hyper_shape=0.0, hyper_rate=0.0, damping=0.1, maximum=1e12)
    with pytest.raises(ValueError, match="must have dtype"):
        uamp_prior_update(mean, pv.double(), old, floor, **kw)
    with pytest.raises(ValueError, match="must have shape"):
        uamp_prior_update(mean[:, :32], pv, old, floor, **kw)
    with pytest.raises(ValueError, match="C-contiguous"):
        uamp_prior_update(mean.t().contiguous().t(), pv, old, floor, **kw)
    with pytest.raises(ValueError, match="CUDA tensor"):
        uamp_prior_update(mean, pv, old, floor.cpu(), **kw)
