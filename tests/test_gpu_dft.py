"""Tensor-core prefix-DFT operator against an FP64 FFT (known answers).

Tolerance: the split-BF16 3-term product with FP32 tensor-core accumulation
stays within 2e-5 relative L2 of the FP64 DFT (measured 5-8e-6).
"""

import numpy as np
import pytest

from gpu_util import need_gpu, rel_l2

torch = pytest.importorskip("torch")

SHAPES = [
    (256, 256, 128, 128, 2),
    (64, 64, 32, 32, 3),
    (40, 32, 20, 16, 2),     # the archived RTX 4090 example shape
    (48, 40, 21, 15, 2),     # odd prefix lengths (unaligned rows)
    (512, 512, 256, 192, 1),
    (192, 256, 77, 101, 1),  # uneven-batch style prefix
]


def _engine(shape, terms):
    from fbme_b200.config import SBLConfig
    from fbme_b200.engine import FBMEEngine

    n1, n2, m1, m2, b = shape
    cfg = SBLConfig.paper_hybrid_uamp(uamp_polish_size=32, dft_terms=terms)
    return FBMEEngine(b, (n1, n2), (m1, m2), cfg, torch.device("cuda:0"))


@pytest.mark.gpu
@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_forward_adjoint_vs_fp64(shape, terms):
    need_gpu()
    n1, n2, m1, m2, b = shape
    eng = _engine(shape, terms)
    rng = np.random.default_rng(7)
    x = (rng.standard_normal((b, n1 * n2)) + 1j * rng.standard_normal((b, n1 * n2))).astype(np.complex64)
    y = (rng.standard_normal((b, m1 * m2)) + 1j * rng.standard_normal((b, m1 * m2))).astype(np.complex64)
    fx = eng.dft_forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ay = eng.dft_adjoint(torch.from_numpy(y).cuda()).cpu().numpy()
    ref_f = np.fft.fft2(x.astype(np.complex128).reshape(b, n1, n2))[:, :m1, :m2].reshape(b, -1)
    ref_a = (np.fft.ifft2(y.astype(np.complex128).reshape(b, m1, m2), s=(n1, n2)) * n1 * n2).reshape(b, -1)
    assert rel_l2(fx, ref_f) < 2e-5
    assert rel_l2(ay, ref_a) < 2e-5
    assert int(eng.out["status"].abs().sum()) == 0


@pytest.mark.gpu
def test_delta_gives_dft_row_and_adjointness():
    """A(delta_n) is the DFT row exp(-2 pi i <m, n/N>); <A x, y> = <x, A^H y>."""
    need_gpu()
    shape = (64, 48, 30, 20, 1)
    n1, n2, m1, m2, _ = shape
    eng = _engine(shape, 3)
    x = np.zeros((1, n1 * n2), np.complex64)
    k1, k2 = 13, 29
    x[0, k1 * n2 + k2] = 1.0
    fx = eng.dft_forward(torch.from_numpy(x).cuda()).cpu().numpy().reshape(m1, m2)
    a1, a2 = np.meshgrid(np.arange(m1), np.arange(m2), indexing="ij")
    row = np.exp(-2j * np.pi * (a1 * k1 / n1 + a2 * k2 / n2))
    assert np.max(np.abs(fx - row)) < 1e-4
    rng = np.random.default_rng(3)
    xr = (rng.standard_normal((1, n1 * n2)) + 1j * rng.standard_normal((1, n1 * n2))).astype(np.complex64)
    yr = (rng.standard_normal((1, m1 * m2)) + 1j * rng.standard_normal((1, m1 * m2))).astype(np.complex64)
    ax = eng.dft_forward(torch.from_numpy(xr).cuda()).cpu().numpy()
    ahy = eng.dft_adjoint(torch.from_numpy(yr).cuda()).cpu().numpy()
    lhs = np.vdot(yr.astype(np.complex128), ax.astype(np.complex128))
    rhs = np.vdot(ahy.astype(np.complex128), xr.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 2e-5


FFT_SHAPES = [
    (512, 512, 256, 192, 1),  # the precision workload's shape
    (256, 256, 128, 128, 2),
    (192, 256, 77, 101, 1),
    (384, 256, 171, 165, 1),
    (64, 64, 32, 32, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", FFT_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_fp32_fft_mode_error_is_that_of_an_fp32_fft(shape):
    """dft_terms=0 runs the operator as FP32 FFTs: its error against an FP64
    DFT is at most twice that of cuFFT in FP32 on the same input."""
    need_gpu()
    n1, n2, m1, m2, b = shape
    eng = _engine(shape, 0)
    rng = np.random.default_rng(8)
    x = (rng.standard_normal((b, n1 * n2)) + 1j * rng.standard_normal((b, n1 * n2))).astype(np.complex64)
    y = (rng.standard_normal((b, m1 * m2)) + 1j * rng.standard_normal((b, m1 * m2))).astype(np.complex64)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    fx = eng.dft_forward(xt).cpu().numpy()
    ay = eng.dft_adjoint(yt).cpu().numpy()
    ref_f = np.fft.fft2(x.astype(np.complex128).reshape(b, n1, n2))[:, :m1, :m2].reshape(b, -1)
    ref_a = (np.fft.ifft2(y.astype(np.complex128).reshape(b, m1, m2), s=(n1, n2)) * n1 * n2).reshape(b, -1)
    cu_f = torch.fft.fft2(xt.view(b, n1, n2))[:, :m1, :m2].reshape(b, -1).cpu().numpy()
    cu_a = (torch.fft.ifft2(yt.view(b, m1, m2), s=(n1, n2)) * (n1 * n2)).reshape(b, -1).cpu().numpy()
    ef, ea = rel_l2(fx, ref_f), rel_l2(ay, ref_a)
    cf, ca = rel_l2(cu_f, ref_f), rel_l2(cu_a, ref_a)
    print(f"{shape}: forward {ef:.2e} (cuFFT FP32 {cf:.2e}), adjoint {ea:.2e} (cuFFT FP32 {ca:.2e})")
    assert ef <= 2 * cf and ea <= 2 * ca
    assert ef < 2e-7 and ea < 2e-7
