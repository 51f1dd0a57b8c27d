"""Known-answer identities behind the device reformulations, checked on the
CPU with the oracle operator:

  * A(delta_n) equals the DFT row; diag(A^H A) = M;
  * the Gram of prefix Fourier atoms is a product of 1-D Dirichlet kernels;
  * A_S^H y equals (A^H y)[S];
  * ||y - A_S mu||^2 = ||y||^2 - 2 Re(c^H mu) + mu^H G mu;
  * A^H(y - A_S mu)[n] = (A^H y)[n] - sum_k mu_k D(n - n_k).
"""

import numpy as np

from oracle import fbme_oracle as O


def _dirichlet(M, N):
    d = np.arange(N)
    return np.exp(2j * np.pi * np.outer(np.arange(M), d) / N).sum(0)


def test_delta_row_and_gram_diagonal():
    op = O.PrefixOperator((24, 20), (10, 7), np.complex128)
    x = np.zeros((1, op.n_grid), complex)
    x[0, 5 * 20 + 3] = 1
    row = op.forward_flat(x)[0].reshape(10, 7)
    a1, a2 = np.meshgrid(np.arange(10), np.arange(7), indexing="ij")
    np.testing.assert_allclose(row, np.exp(-2j * np.pi * (a1 * 5 / 24 + a2 * 3 / 20)), atol=1e-12)
    cols = op.fourier_columns(np.arange(op.n_grid)[None])[0]
    np.testing.assert_allclose(np.sum(np.abs(cols) ** 2, 0), op.n_samples, rtol=1e-12)


def test_dirichlet_gram_column_data_and_residual_identities():
    rng = np.random.default_rng(0)
    n1, n2, m1, m2, k = 32, 40, 13, 17, 9
    op = O.PrefixOperator((n1, n2), (m1, m2), np.complex128)
    S = rng.choice(n1 * n2, k, replace=False)
    A = op.fourier_columns(S[None])[0]
    D1, D2 = _dirichlet(m1, n1), _dirichlet(m2, n2)
    a1, a2 = S // n2, S % n2
    G = D1[(a1[:, None] - a1[None, :]) % n1] * D2[(a2[:, None] - a2[None, :]) % n2]
    np.testing.assert_allclose(G, A.conj().T @ A, atol=1e-9)
    y = rng.standard_normal(m1 * m2) + 1j * rng.standard_normal(m1 * m2)
    bp = op.adjoint_flat(y[None])[0]
    c = bp[S]
    np.testing.assert_allclose(c, A.conj().T @ y, atol=1e-9)
    mu = rng.standard_normal(k) + 1j * rng.standard_normal(k)
    direct = np.sum(np.abs(y - A @ mu) ** 2)
    ident = np.sum(np.abs(y) ** 2) - 2 * np.real(np.vdot(c, mu)) + np.real(np.vdot(mu, G @ mu))
    assert abs(direct - ident) / direct < 1e-10
    r_direct = op.adjoint_flat((y - A @ mu)[None])[0]
    n_1, n_2 = np.divmod(np.arange(n1 * n2), n2)
    acc = np.zeros(n1 * n2, complex)
    for j in range(k):
        acc += mu[j] * D1[(n_1 - a1[j]) % n1] * D2[(n_2 - a2[j]) % n2]
    np.testing.assert_allclose(bp - acc, r_direct, atol=1e-8)


def test_oracle_fp64_close_to_fp32():
    """complex128 input promotes the whole restatement; FP32 stays close."""
    from fbme_b200 import scenes

    s = scenes.config_scene("c1", 4)
    r32 = O.fbme_solve(s.y, s.grid, "stable")
    r64 = O.fbme_solve(s.y.astype(np.complex128), s.grid, "stable")
    x32, x64 = r32["x"].reshape(-1), r64["x"].reshape(-1)
    assert set(np.flatnonzero(x32)) == set(np.flatnonzero(x64))
    assert np.linalg.norm(x32 - x64) / np.linalg.norm(x64) < 1e-4
