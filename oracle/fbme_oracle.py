"""CPU oracle for the FBME plan-replay hot path (numpy restatement).

TEST INFRASTRUCTURE ONLY.  This module is the checker: ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path
(``fbme_b200`` and the drop-in ``torch_sbl`` / ``torch_sbl_fastest_stable``
packages) never imports, calls or falls back to it.

It restates, in plain numpy, the algorithm of the reference package
``torch_sbl`` (FBME-SBL v1.1) for the locked FBME-Fast / FBME-Stable
profiles (``mode="uamp"``) and the ``mode="cg"`` PCG + Hutchinson path.
Every function cites the reference ``file:line`` it follows.  Arithmetic
runs in the dtype of the input (complex64/float32 mirrors the reference's
complex64 run; complex128 gives the FP64 oracle).

Pinning: the restatement is checked against golden vectors produced by
executing the reference itself on seeded synthetic scenes
(``tests/golden/make_golden.py`` writes them; ``tests/test_oracle_golden.py``
compares).  The reference ships no golden vectors of its own.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import ceil, log, prod
from typing import Any

import numpy as np

try:  # scipy is only used for triangular solves; numpy fallback below.
    from scipy.linalg import solve_triangular as _solve_triangular
except Exception:  # pragma: no cover
    _solve_triangular = None


# ---------------------------------------------------------------------------
# Configuration (the subset of torch_sbl/solver.py:34-176 the hot path reads)
# ---------------------------------------------------------------------------


@dataclass
class OracleConfig:
    """Hot-path fields of ``SBLConfig`` (torch_sbl/solver.py:34-176)."""

    max_iter: int = 200
    min_iter: int = 3
    tol: float = 1e-4
    hyper_shape: float = 1e-8
    hyper_rate: float = 1e-8
    noise_shape: float = 1e-8
    noise_rate: float = 1e-8
    initial_noise_fraction: float = 1e-2
    initialization: str = "backprojection"
    initialization_blend: float = 0.1
    fixed_noise_variance: float | None = None
    noise_update: str = "em"
    damping: float = 0.15
    min_variance: float = 1e-12
    max_precision: float = 1e12
    mode: str = "auto"
    dense_threshold: int = 2048
    cg_tolerance: float = 1e-5
    cg_initial_tolerance: float = 1e-2
    cg_max_iter: int = 150
    cg_check_interval: int = 8
    cg_fixed_iterations: int = 0
    cg_preconditioner: str = "low_rank"
    cg_preconditioner_rank: int = 32
    cg_damping: float = 0.9
    hutchinson_probes: int = 32
    max_hutchinson_probes: int = 128
    initial_hutchinson_probes: int = 16
    auto_probe_scaling: bool = True
    adaptive_cg: bool = True
    adaptive_probes: bool = False
    cg_warm_start: bool = True
    cg_min_iter: int = 20
    convergence_patience: int = 2
    convergence_check_interval: int = 2
    cuda_cholesky_jitter_multiplier: float = 8.0
    cg_matvec: str = "tbt"
    uamp_damping: float = 0.1
    uamp_adaptive_damping: bool = True
    uamp_max_damping: float = 0.8
    uamp_min_iter: int = 10
    uamp_auto_iterations: bool = True
    uamp_iteration_offset: float = 10.0
    uamp_iteration_scale: float = 1.1
    uamp_polish_size: int = 0
    uamp_polish_iterations: int = 1
    uamp_polish_prune_tail: bool = False
    uamp_polish_reinitialize: bool = False
    uamp_polish_damping: float = 0.0
    uamp_polish_evidence_gate: bool = False
    uamp_polish_evidence_margin_factor: float = 0.0
    uamp_polish_residual_exchange_size: int = 0
    uamp_polish_fixed_budget_diagnostics: bool = False
    uamp_polish_global_certificate: bool = False
    uamp_polish_support_repairs: int = 0
    uamp_polish_coordinate_tolerance: float = 1e-6
    uamp_polish_familywise_error_rate: float | None = None
    uamp_support_false_alarm_budget: float | None = None
    active_set: bool = True
    active_set_start: int = 30
    active_set_check_interval: int = 2
    active_set_min_size: int = 32
    active_set_max_size: int = 256
    active_set_tail_fraction: float = 5e-2
    seed: int = 0

    @classmethod
    def fast_hybrid_uamp(cls, **overrides: Any) -> "OracleConfig":
        """torch_sbl/solver.py:197-227."""
        s: dict[str, Any] = dict(
            mode="uamp", max_iter=200, min_iter=1, tol=0.0,
            uamp_auto_iterations=True, uamp_min_iter=3,
            uamp_iteration_offset=1.0, uamp_iteration_scale=1.0,
            uamp_polish_size=32, uamp_polish_iterations=2,
            uamp_polish_prune_tail=True, uamp_polish_reinitialize=True,
            uamp_polish_damping=0.0, uamp_polish_evidence_gate=True,
            uamp_polish_residual_exchange_size=0, active_set=False,
        )
        s.update(overrides)
        return cls(**s)

    @classmethod
    def certified_hybrid_uamp(cls, **overrides: Any) -> "OracleConfig":
        """torch_sbl/solver.py:300-316."""
        s: dict[str, Any] = dict(uamp_polish_global_certificate=True, uamp_polish_iterations=4,
                                 uamp_polish_support_repairs=1)
        s.update(overrides)
        return cls.fast_hybrid_uamp(**s)

    @classmethod
    def paper_hybrid_uamp(cls, **overrides: Any) -> "OracleConfig":
        """torch_sbl/solver.py:229-280 (fields that reach the hot path)."""
        s: dict[str, Any] = dict(
            tol=0.0, hyper_shape=0.0, hyper_rate=0.0, noise_shape=0.0,
            noise_rate=0.0, uamp_iteration_offset=0.0,
            uamp_iteration_scale=0.8, uamp_damping=0.05,
            uamp_adaptive_damping=False, uamp_polish_iterations=3,
            uamp_polish_residual_exchange_size=12,
            uamp_polish_evidence_margin_factor=64.0,
            uamp_polish_fixed_budget_diagnostics=True,
            uamp_support_false_alarm_budget=0.5,
        )
        s.update(overrides)
        return cls.fast_hybrid_uamp(**s)

    @classmethod
    def stable(cls, polish_size: int = 32) -> "OracleConfig":
        """FBME-Stable: torch_sbl_fastest_stable/profiles.py:110-115 over
        torch_sbl/cuda_graph.py:148-154 (realtime = paper preset)."""
        return cls.paper_hybrid_uamp(
            uamp_polish_size=polish_size, uamp_polish_iterations=3,
            uamp_polish_residual_exchange_size=12,
            uamp_polish_fixed_budget_diagnostics=True,
        )

    @classmethod
    def fastest(cls, polish_size: int = 32) -> "OracleConfig":
        """FBME-Fast: torch_sbl_fastest_stable/profiles.py:63-70."""
        return cls.paper_hybrid_uamp(
            uamp_polish_size=polish_size, uamp_polish_iterations=2,
            uamp_polish_residual_exchange_size=0,
            uamp_polish_fixed_budget_diagnostics=False,
        )


# ---------------------------------------------------------------------------
# Prefix Fourier operator (torch_sbl/operators.py)
# ---------------------------------------------------------------------------


def _next_smooth_length(minimum: int) -> int:
    """operators.py:10-20."""
    candidate = int(minimum)
    while True:
        r = candidate
        for f in (2, 3, 5, 7):
            while r % f == 0:
                r //= f
        if r == 1:
            return candidate
        candidate += 1


class PrefixOperator:
    """Prefix block of the unnormalised 2-D DFT (operators.py:23-160).

    Coefficients are ``[B, N1*N2]`` (row-major), data ``[B, M1*M2]``.
    """

    def __init__(self, grid, sample, cdtype=np.complex64, observation_mask=None):
        self.grid = tuple(int(v) for v in grid)
        self.sample = tuple(int(v) for v in sample)
        if len(self.grid) != 2 or len(self.sample) != 2:
            raise ValueError("the oracle handles 2-D grids")
        if any(m <= 0 or m > n for m, n in zip(self.sample, self.grid)):
            raise ValueError("Each sample dimension must satisfy 0 < M <= N.")
        self.cdtype = np.dtype(cdtype)
        self.rdtype = np.float64 if self.cdtype == np.complex128 else np.float32
        self.n_grid = prod(self.grid)
        self.full_n_samples = prod(self.sample)
        # observed samples (operators.py:57-75): data hold only those
        self.observed = None
        if observation_mask is not None:
            mask = np.asarray(observation_mask, bool)
            if mask.shape != self.sample:
                raise ValueError(f"observation_mask must have shape {self.sample}, got {mask.shape}.")
            self.observed = np.flatnonzero(mask.reshape(-1))
            if self.observed.size == 0:
                raise ValueError("observation_mask must retain at least one sample.")
        self.n_samples = self.full_n_samples if self.observed is None else int(self.observed.size)
        # operators.py:103-147 embedding for the BTTB (Toeplitz) matvec
        self.embedding = tuple(_next_smooth_length(2 * m - 1) for m in self.sample)
        pos, lag = [], []
        for m, length, n in zip(self.sample, self.embedding, self.grid):
            pos.append(np.concatenate([np.arange(m), np.arange(length - m + 1, length)]))
            lag.append(np.concatenate([np.arange(m), np.arange(-(m - 1), 0)]))
        p0, p1 = np.meshgrid(pos[0], pos[1], indexing="ij")
        l0, l1 = np.meshgrid(lag[0], lag[1], indexing="ij")
        self.embedding_positions = (p0 * self.embedding[1] + p1).reshape(-1)
        self.embedding_lags = (
            np.remainder(l0, self.grid[0]) * self.grid[1] + np.remainder(l1, self.grid[1])
        ).reshape(-1)
        a0, a1 = np.meshgrid(np.arange(self.sample[0]), np.arange(self.sample[1]), indexing="ij")
        self.sample_coordinates = np.stack([a0.reshape(-1), a1.reshape(-1)], 1)
        if self.observed is not None:
            self.sample_coordinates = self.sample_coordinates[self.observed]

    def restrict(self, full: np.ndarray) -> np.ndarray:
        """operators.py:473-482: observed entries of [B, M1*M2, ...] data."""
        return full if self.observed is None else full[:, self.observed]

    def expand(self, data: np.ndarray) -> np.ndarray:
        """operators.py:484-496: observed entries scattered into a zero block."""
        if self.observed is None:
            return data
        full = np.zeros((data.shape[0], self.full_n_samples, *data.shape[2:]), data.dtype)
        full[:, self.observed] = data
        return full

    def forward_flat(self, coefficients: np.ndarray) -> np.ndarray:
        """operators.py:237-253: fft2 then crop (and restrict)."""
        b = coefficients.shape[0]
        field = coefficients.reshape(b, *self.grid)
        spec = np.fft.fft2(field, axes=(1, 2))
        full = spec[:, : self.sample[0], : self.sample[1]].reshape(b, self.full_n_samples)
        return self.restrict(full).astype(self.cdtype)

    def adjoint_flat(self, data: np.ndarray) -> np.ndarray:
        """operators.py:255-280: N * ifft2 with end zero padding."""
        b = data.shape[0]
        field = self.expand(data).reshape(b, *self.sample)
        coeff = np.fft.ifft2(field, s=self.grid, axes=(1, 2)).astype(self.cdtype)
        return (coeff * self.rdtype(self.n_grid)).reshape(b, self.n_grid)

    def fourier_columns(self, flat_indices: np.ndarray) -> np.ndarray:
        """operators.py:444-466: exp(-2*pi*i*<m, n/N>) for selected atoms.

        Follows the reference's real-dtype phase arithmetic (phase formed
        in the real dtype, then the complex exponential).
        """
        rd = self.rdtype
        n1 = (flat_indices // self.grid[1]).astype(rd)
        n2 = (flat_indices % self.grid[1]).astype(rd)
        c = self.sample_coordinates.astype(rd) / np.array(self.grid, dtype=rd)
        phase = c[None, :, 0:1] * n1[:, None, :] + c[None, :, 1:2] * n2[:, None, :]
        arg = (rd(-2.0 * np.pi) * phase).astype(rd)
        return np.exp(1j * arg).astype(self.cdtype)

    def toeplitz_spectrum(self, prior: np.ndarray, noise: np.ndarray) -> np.ndarray:
        """operators.py:299-326: BTTB embedding spectrum of
        Q = noise*I + A diag(prior) A^H."""
        b = prior.shape[0]
        field = prior.astype(self.cdtype).reshape(b, *self.grid)
        lags = np.fft.fft2(field, axes=(1, 2)).astype(self.cdtype).reshape(b, self.n_grid)
        kernel = np.zeros((b, prod(self.embedding)), self.cdtype)
        kernel[:, self.embedding_positions] = lags[:, self.embedding_lags]
        kernel[:, 0] += noise
        return np.fft.fft2(kernel.reshape(b, *self.embedding), axes=(1, 2)).astype(self.cdtype)

    def toeplitz_matvec(self, data: np.ndarray, spectrum: np.ndarray) -> np.ndarray:
        """operators.py:328-355: data [B, M, R] -> Q data."""
        b, _, r = data.shape
        field = data.reshape(b, *self.sample, r)
        tr = np.fft.fft2(field, s=self.embedding, axes=(1, 2)).astype(self.cdtype)
        prod_ = np.fft.ifft2(tr * spectrum[..., None], axes=(1, 2)).astype(self.cdtype)
        return prod_[:, : self.sample[0], : self.sample[1], :].reshape(b, self.n_samples, r)

    def adjoint(self, data: np.ndarray) -> np.ndarray:
        """operators.py:219-235: [B, M, R] -> [B, N, R]."""
        b, _, r = data.shape
        field = data.reshape(b, *self.sample, r)
        coeff = np.fft.ifft2(field, s=self.grid, axes=(1, 2)).astype(self.cdtype)
        return (coeff * self.rdtype(self.n_grid)).reshape(b, self.n_grid, r)

    def forward(self, coeff: np.ndarray) -> np.ndarray:
        """operators.py:208-217: [B, N, R] -> [B, M, R]."""
        b, _, r = coeff.shape
        spec = np.fft.fft2(coeff.reshape(b, *self.grid, r), axes=(1, 2)).astype(self.cdtype)
        return spec[:, : self.sample[0], : self.sample[1], :].reshape(b, self.n_samples, r)


# ---------------------------------------------------------------------------
# Small helpers
# ---------------------------------------------------------------------------


def _finfo(rd):
    fi = np.finfo(rd)
    return rd(fi.eps), rd(fi.tiny)


def _abs2(z: np.ndarray) -> np.ndarray:
    """``z.abs().square()`` in the real dtype of ``z``."""
    return np.square(np.abs(z))


def _tri_solve(lower: np.ndarray, rhs: np.ndarray, *, upper: bool = False) -> np.ndarray:
    """Batched triangular solve (torch.linalg.solve_triangular)."""
    out = np.empty(np.broadcast_shapes(lower.shape[:-2], rhs.shape[:-2]) + rhs.shape[-2:], rhs.dtype)
    for i in range(out.shape[0]):
        a = lower[i]
        if _solve_triangular is not None:
            out[i] = _solve_triangular(a, rhs[i], lower=not upper, check_finite=False)
        else:  # pragma: no cover
            out[i] = np.linalg.solve(a, rhs[i])
    return out


def _stable_cholesky(matrix: np.ndarray, tiny, eps, *, mode: str, multiplier: float,
                     fallback=(1.0, 10.0, 1e2, 1e3, 1e4, 1e5)):
    """solver.py:2898-2931 (_stable_cholesky_raw).

    ``mode="cuda"``: one deterministic loading ``multiplier*eps*scale``
    (solver.py:2910-2920).  ``mode="cpu"``: the first loading of
    ``fallback`` that factors (solver.py:2922-2931).
    """
    k = matrix.shape[-1]
    eye = np.eye(k, dtype=matrix.dtype)
    scale = np.abs(np.real(np.diagonal(matrix, axis1=-2, axis2=-1))).mean(axis=1)
    scale = np.maximum(scale, tiny).astype(type(eps))
    base = eps * scale
    mults = (multiplier,) if mode == "cuda" else fallback
    for mlt in mults:
        loaded = matrix + (type(eps)(mlt) * base)[:, None, None] * eye
        try:
            return np.linalg.cholesky(loaded)
        except np.linalg.LinAlgError:
            if mode == "cuda":
                raise RuntimeError("CUDA Cholesky failed after deterministic diagonal loading.")
    return None


# ---------------------------------------------------------------------------
# Reduced exact posterior with evidence (solver.py:3591-3779)
# ---------------------------------------------------------------------------


def active_posterior_with_evidence(y, prior, noise, op: PrefixOperator, active, *, columns,
                                   gram, column_data, data_energy, chol_mode, chol_multiplier,
                                   tail_loading=0.0, certificate=False):
    """solver.py:3591-3779; with ``certificate`` the inactive-atom
    certificate of the result (3757-3770) is returned as a fifth value.

    ``tail_loading``: 0 (the exact zero-tail model of the polish) or None,
    the omitted prior variance sum(prior) - sum(prior[active]) as an
    isotropic loading (solver.py:3632-3639, the cg active-set posterior).
    Returns (mean[B,N], posterior_variance[B,N], data_diagonal[B,N], nle[B]).
    """
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    b, k = active.shape
    rows = np.arange(b)[:, None]
    gamma = prior[rows, active]
    if tail_loading is None:
        omitted = np.maximum(prior.sum(axis=1, dtype=rd) - gamma.sum(axis=1, dtype=rd), rd(0.0))
    else:
        omitted = rd(tail_loading)
    eff_noise = (noise + omitted).astype(rd)
    system = np.zeros((b, k, k), y.dtype)
    system[:, np.arange(k), np.arange(k)] = (rd(1.0) / gamma).astype(y.dtype)
    system = system + gram / eff_noise[:, None, None]
    system = rd(0.5) * (system + np.conj(np.swapaxes(system, 1, 2)))
    dscale = np.sqrt(np.maximum(np.real(np.diagonal(system, axis1=1, axis2=2)), tiny))
    eq = system / dscale[:, :, None] / dscale[:, None, :]
    eq = rd(0.5) * (eq + np.conj(np.swapaxes(eq, 1, 2)))
    chol = _stable_cholesky(eq, tiny, eps, mode=chol_mode, multiplier=chol_multiplier)
    if chol is None:
        raise RuntimeError("Reduced active-set posterior is not positive definite.")
    rhs = column_data / eff_noise[:, None, None]
    srhs = rhs / dscale[:, :, None]
    fwd = _tri_solve(chol, srhs)
    eq_mean = _tri_solve(np.conj(np.swapaxes(chol, 1, 2)), fwd, upper=True)
    inv_factor = _tri_solve(chol, np.broadcast_to(np.eye(k, dtype=y.dtype), (b, k, k)))
    eq_var = _abs2(inv_factor).sum(axis=1)
    a_mean = (eq_mean / dscale[:, :, None])[:, :, 0]
    a_var = np.maximum(np.real(eq_var / np.square(dscale)), rd(0.0)).astype(rd)
    a_dd = np.maximum((gamma - a_var) / np.square(gamma), rd(0.0))
    logdet_sys = rd(2.0) * (
        np.log(np.maximum(np.real(np.diagonal(chol, axis1=1, axis2=2)), tiny)).sum(axis=1)
        + np.log(dscale).sum(axis=1)
    )
    logdet = rd(op.n_samples) * np.log(eff_noise) + np.log(gamma).sum(axis=1) + logdet_sys
    quad = np.maximum(
        data_energy / eff_noise - np.real((np.conj(rhs[:, :, 0]) * a_mean).sum(axis=1)), rd(0.0)
    )
    nle = (logdet + quad).astype(rd)
    mean = np.zeros((b, op.n_grid), y.dtype)
    pv = prior.copy()
    dd = np.zeros_like(prior)
    mean[rows, active] = a_mean
    pv[rows, active] = a_var
    dd[rows, active] = a_dd
    if certificate:
        cert = inactive_evidence_certificate(y, columns, a_mean, eff_noise, dscale, chol, op, active)
        return mean, pv, dd, nle, cert
    return mean, pv, dd, nle


def ratio_threshold_for_evidence_tolerance(tolerance: float) -> float:
    """solver.py:3499-3519: the rho >= 1 with rho - 1 - log(rho) = tolerance,
    by doubling an upper bound and 64 bisection steps."""
    if tolerance <= 0.0:
        return 1.0
    lo, hi = 1.0, 2.0
    while hi - 1.0 - log(hi) < tolerance:
        hi *= 2.0
    for _ in range(64):
        mid = 0.5 * (lo + hi)
        if mid - 1.0 - log(mid) < tolerance:
            lo = mid
        else:
            hi = mid
    return hi


def inactive_evidence_certificate(y, columns, a_mean, eff_noise, dscale, chol, op: PrefixOperator, active):
    """solver.py:3522-3588: for every atom j, q_j = a_j^H C^-1 y (one adjoint
    transform of the residual / noise) and s_j = a_j^H C^-1 a_j = M / nu -
    ||L^-1 D^-1 A_S^H a_j||^2 / nu^2; the best inactive ratio |q_j|^2 / s_j
    with its one-coordinate evidence gain and optimal variance."""
    rd = op.rdtype
    _, tiny = _finfo(rd)
    b, k = active.shape
    rows = np.arange(b)[:, None]
    residual = y - (columns @ a_mean[:, :, None])[:, :, 0]
    q = op.adjoint_flat(residual / eff_noise[:, None])
    m = columns.shape[1]
    cross = np.conj(op.adjoint_flat(np.swapaxes(columns, 1, 2).reshape(b * k, m))).reshape(b, k, -1)
    solved = _tri_solve(chol, cross / dscale[:, :, None])
    reduction = _abs2(solved).sum(axis=1, dtype=rd)
    precision = np.maximum(rd(op.n_samples) / eff_noise[:, None] - reduction / np.square(eff_noise)[:, None],
                           tiny).astype(rd)
    ratio = (_abs2(q) / precision).astype(rd)
    ratio[rows, active] = 0
    best = np.argmax(ratio, axis=1)
    max_ratio = ratio[np.arange(b), best]
    best_prec = precision[np.arange(b), best]
    up = max_ratio > 1.0
    gain = np.where(up, max_ratio - rd(1.0) - np.log(np.maximum(max_ratio, tiny)), rd(0.0)).astype(rd)
    optvar = np.where(up, (max_ratio - rd(1.0)) / best_prec, rd(0.0)).astype(rd)
    return dict(max_ratio=max_ratio, best_index=best.astype(np.int64), evidence_gain=gain,
                optimal_variance=optvar)


def active_evidence_certificate(a_mean, a_pv, a_gamma, active):
    """solver.py:3219-3317: the best exact one-coordinate update among the
    active atoms (leave-one-out statistics by Sherman-Morrison)."""
    rd = a_pv.dtype.type
    _, tiny = _finfo(rd)
    b = a_pv.shape[0]
    r = np.arange(b)
    g = np.maximum(a_gamma, tiny)
    q = a_mean / g
    s = np.maximum((g - a_pv) / np.square(g), tiny)
    down = np.clip(a_pv / g, tiny, rd(1.0))
    loo = np.maximum(s / down, tiny)
    ratio = _abs2(q) / np.maximum(s * down, tiny)
    optvar = np.where(ratio > 1.0, (ratio - rd(1.0)) / loo, rd(0.0)).astype(rd)
    current = (-np.log(down) - g * _abs2(q) / down).astype(rd)
    optimal = np.where(ratio > 1.0, np.log(np.maximum(ratio, tiny)) - ratio + rd(1.0), rd(0.0))
    gain = np.maximum(current - optimal, rd(0.0)).astype(rd)
    pos = np.argmax(gain, axis=1)
    nondel = np.where(optvar > 0.0, gain, rd(0.0))
    npos = np.argmax(nondel, axis=1)
    dpos = np.argmax(current, axis=1)
    return dict(max_gain=gain[r, pos], best_position=pos, best_index=active[r, pos].astype(np.int64),
                optimal_variance=optvar[r, pos], max_nondeletion_gain=nondel[r, npos],
                max_deletion_gain=current[r, dpos], best_deletion_position=dpos)


def active_evidence_deletion_gain(a_mean, a_pv, a_gamma):
    """solver.py:3219-3317: the ``deletion_gain`` (current_delta) field."""
    rd = a_pv.dtype.type
    _, tiny = _finfo(rd)
    g = np.maximum(a_gamma, tiny)
    q = a_mean / g
    s = np.maximum((g - a_pv) / np.square(g), tiny)
    down = np.clip(a_pv / g, tiny, rd(1.0))
    return (-np.log(down) - g * _abs2(q) / down).astype(rd)


# ---------------------------------------------------------------------------
# UAMP sweep (solver.py:2726-2870, torch branch 2808-2850; Triton kernels
# triton_kernels.py:37-192 compute the same expressions)
# ---------------------------------------------------------------------------


@dataclass
class UAMPState:
    """solver.py:795-804."""

    mean: np.ndarray
    variance: np.ndarray
    message: np.ndarray
    prediction: np.ndarray
    data_variance: np.ndarray


def uamp_sweep(y, prior, noise, op, st: UAMPState, *, damping, initial_backprojection=None,
               compute_prediction=True, prior_floor=None, prior_damping=0.0,
               prior_maximum=1e12, hyper_shape=0.0, hyper_rate=0.0):
    """One UAMP iteration.  Returns (mean, var, dof, new_state, next_prior).

    ``prior_floor`` given: fused ARD update of triton_kernels.py:163-184.
    """
    rd = op.rdtype
    _, tiny = _finfo(rd)
    d = rd(damping)
    cv = np.maximum(st.variance, tiny)
    dv = np.maximum(st.data_variance, tiny)
    # message (triton_kernels.py:72-89; solver.py:2810-2818)
    precision = rd(1.0) / (dv + noise)
    pseudo_data = st.prediction - dv[:, None] * st.message
    cand = precision[:, None] * (y - pseudo_data)
    message = d * st.message + (rd(1.0) - d) * cand
    pv = np.maximum((dv + noise) / rd(op.n_samples), tiny)
    if initial_backprojection is not None:
        lifted = initial_backprojection * ((rd(1.0) - d) / (dv + noise))[:, None]
    else:
        lifted = op.adjoint_flat(message)
    # denoise (triton_kernels.py:140-158; solver.py:2832-2850)
    denom = np.maximum(prior + pv[:, None], tiny)
    gain = prior / denom
    pseudo_mean = st.mean + pv[:, None] * lifted
    cand_mean = gain * pseudo_mean
    cand_var = prior * pv[:, None] / denom
    mean = d * st.mean + (rd(1.0) - d) * cand_mean
    var = np.maximum(d * cv + (rd(1.0) - d) * cand_var, tiny)
    dof = np.clip(rd(1.0) - var / np.maximum(prior, tiny), 0, 1).sum(axis=1, dtype=rd)
    next_dv = var.sum(axis=1, dtype=rd)
    next_prior = None
    if prior_floor is not None:
        # triton_kernels.py:163-184 (== solver.py:1630-1648 + 1783-1787)
        second = _abs2(mean) + var
        cp = (second + rd(hyper_rate)) / rd(1.0 + hyper_shape)
        cp = np.maximum(prior_floor[:, None], np.minimum(rd(prior_maximum), cp))
        nxt = rd(prior_damping) * prior + rd(1.0 - prior_damping) * cp
        next_prior = np.maximum(nxt, prior_floor[:, None])
    prediction = op.forward_flat(mean) if compute_prediction else st.prediction
    return mean, var, dof, UAMPState(mean, var, message, prediction, next_dv), next_prior


# ---------------------------------------------------------------------------
# fast_sbl, mode="uamp" (solver.py:925-2393, plan-relevant branches)
# ---------------------------------------------------------------------------


def _uamp_iteration_limit(cfg: OracleConfig, n_grid: int, n_samples: int) -> int:
    """solver.py:1287-1309."""
    minimum = max(cfg.min_iter, cfg.uamp_min_iter)
    limit = cfg.max_iter
    if cfg.uamp_auto_iterations:
        budget = ceil(cfg.uamp_iteration_offset + cfg.uamp_iteration_scale * n_grid / n_samples)
        limit = min(cfg.max_iter, max(minimum, budget))
    return limit


def fast_sbl_uamp(data: np.ndarray, grid, cfg: OracleConfig, *, chol_mode: str = "cuda",
                  stop_after_uamp: bool = False, initial_prior: np.ndarray | None = None,
                  observation_mask: np.ndarray | None = None):
    """Restatement of ``fast_sbl`` for ``mode="uamp"`` with the polish.

    ``data`` is ``[M1, M2]`` or ``[B, M1, M2]``.  Returns a dict of the
    ``SBLResult`` fields the FBME plans fill (solver.py:2154-2393).
    ``initial_prior`` ([B, N], optional) replaces the initial prior variances
    of solver.py:1072-1099 (floored as there): the warm start of the learned
    path; everything else is unchanged.
    """
    data = np.asarray(data)
    cdtype = np.complex128 if data.dtype in (np.complex128, np.float64) else np.complex64
    single = data.ndim == 2
    y3 = data[None] if single else data
    b = y3.shape[0]
    sample = y3.shape[1:]
    op = PrefixOperator(grid, sample, cdtype, observation_mask)
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    y = op.restrict(y3.reshape(b, op.full_n_samples)).astype(cdtype)  # solver.py:1022-1024
    n, m = op.n_grid, op.n_samples
    if cfg.uamp_support_false_alarm_budget is not None and cfg.uamp_support_false_alarm_budget >= n:
        raise ValueError("uamp_support_false_alarm_budget must be smaller than the grid size.")

    # initialisation (solver.py:1063-1099, 1151-1182)
    data_power = np.maximum(_abs2(y).mean(axis=1, dtype=rd), eps).astype(rd)
    variance_floor = np.maximum(data_power * rd(cfg.min_variance), tiny).astype(rd)
    uniform = data_power[:, None] / rd(n)
    initial_bp = None
    if cfg.initialization == "backprojection":
        bp = op.adjoint_flat(y)
        initial_bp = bp
        e = _abs2(bp)
        structured = e / np.maximum(e.sum(axis=1, keepdims=True, dtype=rd), eps) * data_power[:, None]
        prior = rd(cfg.initialization_blend) * structured + rd(1.0 - cfg.initialization_blend) * uniform
    else:
        prior = np.broadcast_to(uniform, (b, n)).copy()
    prior_floor = variance_floor
    if initial_prior is not None:
        prior = np.asarray(initial_prior, dtype=rd).reshape(b, n)
    prior = np.maximum(prior, prior_floor[:, None]).astype(rd)
    if cfg.fixed_noise_variance is None:
        noise = np.maximum(rd(cfg.initial_noise_fraction) * data_power, variance_floor).astype(rd)
    else:
        noise = np.full(b, cfg.fixed_noise_variance, rd)
    st = UAMPState(np.zeros((b, n), cdtype), prior.copy(), np.zeros((b, m), cdtype),
                   np.zeros((b, m), cdtype), prior.sum(axis=1, dtype=rd))
    damping = cfg.uamp_damping
    if cfg.uamp_adaptive_damping:
        damping = max(damping, min(cfg.uamp_max_damping, 0.02 * n / m))
    limit = _uamp_iteration_limit(cfg, n, m)
    keep = rd(cfg.damping)

    # EM loop (solver.py:1315-1798 for mode="uamp", fused Triton updates)
    for it in range(1, limit + 1):
        mean, var, dof_u, st, next_prior = uamp_sweep(
            y, prior, noise, op, st, damping=damping,
            initial_backprojection=initial_bp if it == 1 else None,
            prior_floor=prior_floor, prior_damping=cfg.damping,
            prior_maximum=cfg.max_precision, hyper_shape=cfg.hyper_shape,
            hyper_rate=cfg.hyper_rate)
        dof = np.minimum(dof_u, rd(m * (1.0 - 10.0 * float(eps))))
        new_prior = next_prior
        # noise update (triton_kernels.py:298-318; solver.py:1751-1768)
        if cfg.fixed_noise_variance is None:
            energy = _abs2(y - st.prediction).sum(axis=1, dtype=rd)
            if cfg.noise_update == "em":
                cand = (energy + noise * dof + rd(cfg.noise_rate)) / rd(m + cfg.noise_shape)
            else:
                cand = (energy + rd(cfg.noise_rate)) / np.maximum(rd(m) - dof + rd(cfg.noise_shape), eps)
            cand = np.maximum(cand, variance_floor)
            new_noise = keep * noise + (rd(1.0) - keep) * cand
            new_noise = np.maximum(new_noise, variance_floor)
            noise = new_noise.astype(rd)
        prior = np.maximum(new_prior, prior_floor[:, None]).astype(rd)

    # final E-step (solver.py:1907-1925)
    mean, var, dof_u, st, _ = uamp_sweep(y, prior, noise, op, st, damping=damping,
                                         compute_prediction=False)
    if stop_after_uamp:
        # state after the final E-step (before top-K and the polish)
        return dict(mean=mean, variance=var, prior_variance=prior, noise_variance=noise,
                    backprojection=initial_bp, prediction=st.prediction, iterations=limit,
                    score=_abs2(mean) + var)
    out: dict[str, Any] = {}
    if cfg.uamp_polish_size > 0:
        k = min(cfg.uamp_polish_size, n)
        score = _abs2(mean) + var
        active = _topk_indices(score, k)
        out["uamp_active_indices"] = active.copy()
        out["uamp_score"] = score
        pol = uamp_active_em_polish(y, mean, var, prior, noise, op, active, prior_floor, cfg,
                                    chol_mode=chol_mode)
        mean, var, dd, prior, noise = pol["mean"], pol["pv"], pol["dd"], pol["prior"], pol["noise"]
        out.update({kk: v for kk, v in pol.items() if kk not in ("mean", "pv", "dd", "prior", "noise")})
        if cfg.uamp_polish_fixed_budget_diagnostics:
            gres, nres = fixed_budget_em_residuals(y, mean, var, prior, noise, pol["active_indices"],
                                                   prior_floor, op, cfg)
            trace = pol["evidence_trace"]
            finite = np.isfinite(trace).all(axis=1)
            nonincreasing = (trace[:, 1:] <= trace[:, :-1]).all(axis=1)
            out["fixed_budget_gamma_residual"] = gres
            out["fixed_budget_noise_residual"] = nres
            out["fixed_budget_monotone"] = finite & nonincreasing
            out["fixed_budget_objective_decrease"] = np.maximum(trace[:, 0] - trace[:, -1], rd(0.0))
        # effective DOF from the exact posterior (solver.py:2081-2092, 3156-3181)
        rel = np.clip(prior * dd, 0, 1)
        raw = rel.sum(axis=1, dtype=rd)
        max_dof = rd(m * (1.0 - 10.0 * float(eps)))
        scale = np.minimum(rd(1.0), max_dof / np.maximum(raw, eps))
        dof = (rel * scale[:, None]).sum(axis=1, dtype=rd)
    else:
        dof = np.minimum(dof_u, rd(m * (1.0 - 10.0 * float(eps))))
    precision = (rd(1.0) / prior).astype(rd)
    # support mask (solver.py:2108-2126)
    if cfg.uamp_support_false_alarm_budget is not None:
        thr = rd(log(n / cfg.uamp_support_false_alarm_budget))
        sscore = _abs2(mean) / np.maximum(var, tiny)
        out["support_mask"] = (sscore > thr).reshape((-1,) + tuple(grid))
        out["support_score_threshold"] = np.full(b, thr, rd)
    shape = tuple(grid)
    out.update(
        x=mean.reshape((b,) + shape), posterior_variance=var.reshape((b,) + shape),
        precision=precision.reshape((b,) + shape), noise_variance=noise, effective_dof=dof,
        iterations=limit, mode="uamp", arithmetic_dtype=str(np.dtype(cdtype)),
        active_set_size=(min(cfg.uamp_polish_size, n) if cfg.uamp_polish_size > 0 else 0),
    )
    if single:
        for key, val in list(out.items()):
            if isinstance(val, np.ndarray) and val.ndim >= 1 and val.shape[0] == 1 and key not in (
                    "evidence_trace", "penalized_evidence_trace"):
                out[key] = val[0]
    return out


def _topk_indices(score: np.ndarray, k: int) -> np.ndarray:
    """``torch.topk(score, k).indices``: descending, ties by lower index."""
    order = np.argsort(-score, axis=1, kind="stable")
    return order[:, :k].astype(np.int64)


def uamp_active_em_polish(y, uamp_mean, uamp_var, prior, noise, op, active, prior_floor,
                          cfg: OracleConfig, *, chol_mode="cuda"):
    """solver.py:3961-4510 (branches reachable from the FBME plans)."""
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    b, k = active.shape
    rows = np.arange(b)[:, None]
    m = op.n_samples
    # prune + reinitialise (4079-4106)
    working = prior.copy()
    if cfg.uamp_polish_prune_tail:
        working = np.broadcast_to(prior_floor[:, None], prior.shape).copy()
        working[rows, active] = prior[rows, active]
    if cfg.uamp_polish_reinitialize:
        second = _abs2(uamp_mean) + uamp_var
        working[rows, active] = np.maximum(second[rows, active], prior_floor[:, None])
    columns = op.fourier_columns(active)
    gram = np.conj(np.swapaxes(columns, 1, 2)) @ columns
    column_data = np.conj(np.swapaxes(columns, 1, 2)) @ y[:, :, None]
    data_energy = _abs2(y).sum(axis=1, dtype=rd)
    active_noise = noise.copy()
    best = None
    accepted = []
    pending = None
    exch_acc = np.zeros(b, np.int64) if cfg.uamp_polish_residual_exchange_size > 0 else None
    mean = uamp_mean
    pv = uamp_var
    gcert = cfg.uamp_polish_global_certificate
    for p in range(cfg.uamp_polish_iterations):
        ev = active_posterior_with_evidence(
            y, working, active_noise, op, active, columns=columns, gram=gram,
            column_data=column_data, data_energy=data_energy, chol_mode=chol_mode,
            chol_multiplier=cfg.cuda_cholesky_jitter_multiplier, certificate=gcert)
        c_mean, c_pv, c_dd, c_nle = ev[:4]
        cand = dict(mean=c_mean, pv=c_pv, dd=c_dd, prior=working, noise=active_noise, nle=c_nle,
                    active=active, columns=columns, gram=gram, column_data=column_data)
        if gcert:  # the certificate follows its candidate through the gate (4165-4260)
            cand.update({"cert_" + kk: v for kk, v in ev[4].items()})
        if cfg.uamp_polish_evidence_gate:
            if best is None:
                best = {kk: (v.copy() if isinstance(v, np.ndarray) else v) for kk, v in cand.items()}
            else:
                margin = rd(cfg.uamp_polish_evidence_margin_factor) * eps * (
                    rd(1.0) + np.abs(c_nle) + np.abs(best["nle"]))
                accept = np.isfinite(c_nle) & (~np.isfinite(best["nle"]) | (c_nle <= best["nle"] - margin))
                for key, val in cand.items():
                    mask = accept.reshape((b,) + (1,) * (np.ndim(val) - 1))
                    best[key] = np.where(mask, val, best[key])
                if pending is not None and exch_acc is not None:
                    exch_acc = exch_acc + (accept & pending).astype(np.int64)
                    pending = None
            cur = best
        else:
            cur = cand
        accepted.append(cur["nle"].copy())
        mean, pv, base_prior, base_noise = cur["mean"], cur["pv"], cur["prior"], cur["noise"]
        active, columns, gram, column_data = cur["active"], cur["columns"], cur["gram"], cur["column_data"]
        if p + 1 == cfg.uamp_polish_iterations:
            break
        # EM between evaluations (4320-4391)
        a_gamma = base_prior[rows, active]
        a_pv = pv[rows, active]
        a_mean = mean[rows, active]
        new_g = np.minimum(np.maximum(_abs2(a_mean) + a_pv, prior_floor[:, None]), rd(cfg.max_precision))
        keep = rd(cfg.uamp_polish_damping)
        upd_g = keep * a_gamma + (rd(1.0) - keep) * new_g
        prediction = (columns @ a_mean[:, :, None])[:, :, 0]
        residual = y - prediction
        r_energy = _abs2(residual).sum(axis=1, dtype=rd)
        eff_noise = base_noise
        dof = np.clip(rd(1.0) - a_pv / np.maximum(a_gamma, tiny), 0, 1).sum(axis=1, dtype=rd)
        if cfg.fixed_noise_variance is not None:
            upd_noise = np.full(b, cfg.fixed_noise_variance, rd)
        elif cfg.noise_update == "em":
            upd_noise = (r_energy + eff_noise * dof + rd(cfg.noise_rate)) / rd(m + cfg.noise_shape)
        else:
            upd_noise = (r_energy + rd(cfg.noise_rate)) / np.maximum(rd(m) - dof + rd(cfg.noise_shape), eps)
        upd_noise = np.maximum(upd_noise, prior_floor)
        if cfg.fixed_noise_variance is None:
            active_noise = (keep * base_noise + (rd(1.0) - keep) * upd_noise).astype(rd)
        else:
            active_noise = upd_noise.astype(rd)
        working = base_prior.copy()
        working[rows, active] = upd_g
        ex = min(cfg.uamp_polish_residual_exchange_size, max(k - 1, 0), op.n_grid - k)
        if ex > 0 and p == 0:
            # residual support exchange (4397-4494)
            rscore = _abs2(op.adjoint_flat(residual))
            rscore[rows, active] = -np.inf
            add_idx = _topk_indices(rscore, ex)
            add_energy = rscore[rows, add_idx]
            deletion = active_evidence_deletion_gain(a_mean, a_pv, a_gamma)
            rem_pos = _topk_indices(deletion, ex)
            rem_idx = active[rows, rem_pos]
            ce = rd(float(m))
            ratio = add_energy / np.maximum(base_noise[:, None] * ce, tiny)
            add_gain = np.where(ratio > 1.0, ratio - rd(1.0) - np.log(np.maximum(ratio, tiny)), rd(0.0))
            del_gain = deletion[rows, rem_pos]
            xmask = (add_gain + del_gain) > 0.0
            repl = np.where(xmask, add_idx, rem_idx)
            new_active = active.copy()
            new_active[rows, rem_pos] = repl
            add_gamma = np.maximum(add_energy - base_noise[:, None] * ce, rd(0.0)) / (ce * ce)
            add_gamma = np.minimum(np.maximum(add_gamma, prior_floor[:, None]), rd(cfg.max_precision))
            retained = working[rows, rem_idx]
            working[rows, rem_idx] = np.where(xmask, prior_floor[:, None], retained)
            working[rows, repl] = np.where(xmask, add_gamma, retained)
            active = new_active
            columns = op.fourier_columns(active)
            gram = np.conj(np.swapaxes(columns, 1, 2)) @ columns
            column_data = np.conj(np.swapaxes(columns, 1, 2)) @ y[:, :, None]
            pending = xmask.any(axis=1)
            out_ex = dict(add_idx=add_idx, rem_pos=rem_pos, xmask=xmask)
    fin = best if cfg.uamp_polish_evidence_gate else cand
    dd = cur["dd"]
    f_prior, f_noise, f_active, f_nle = fin["prior"], fin["noise"], fin["active"], fin["nle"]
    cert = {kk[5:]: v for kk, v in fin.items() if kk.startswith("cert_")} if gcert else None
    # support repairs (4511-4628): the best inactive atom replaces the active
    # atom of largest deletion gain; kept when the exact evidence does not rise
    if cfg.uamp_polish_support_repairs > 0 and exch_acc is None:
        exch_acc = np.zeros(b, np.int64)
    for _ in range(cfg.uamp_polish_support_repairs):
        acert = active_evidence_certificate(mean[rows, f_active], pv[rows, f_active],
                                            f_prior[rows, f_active], f_active)
        r = np.arange(b)
        rep_idx = cert["best_index"]
        pos = acert["best_deletion_position"]
        replaced = f_active[r, pos]
        rep_active = f_active.copy()
        rep_active[r, pos] = rep_idx
        rep_prior = f_prior.copy()
        rep_prior[r, replaced] = prior_floor
        rep_prior[r, rep_idx] = np.maximum(cert["optimal_variance"], prior_floor)
        cols = op.fourier_columns(rep_active)
        ch = np.conj(np.swapaxes(cols, 1, 2))
        r_mean, r_pv, r_dd, r_nle, r_cert = active_posterior_with_evidence(
            y, rep_prior, f_noise, op, rep_active, columns=cols, gram=ch @ cols,
            column_data=ch @ y[:, :, None], data_energy=data_energy, chol_mode=chol_mode,
            chol_multiplier=cfg.cuda_cholesky_jitter_multiplier, certificate=True)
        acc = (cert["max_ratio"] > 1.0) & np.isfinite(r_nle) & (r_nle <= f_nle)
        exch_acc = exch_acc + acc.astype(np.int64)
        m2 = acc[:, None]
        mean, pv, dd = np.where(m2, r_mean, mean), np.where(m2, r_pv, pv), np.where(m2, r_dd, dd)
        f_prior = np.where(m2, rep_prior, f_prior)
        f_active = np.where(m2, rep_active, f_active)
        f_nle = np.where(acc, r_nle, f_nle).astype(rd)
        accepted.append(f_nle.copy())
        cert = {kk: np.where(acc, r_cert[kk], v) for kk, v in cert.items()}
    trace = np.stack(accepted, axis=1)
    res = dict(
        mean=mean, pv=pv, dd=dd, prior=f_prior, noise=f_noise,
        negative_log_evidence=f_nle, evidence_trace=trace,
        penalized_negative_log_evidence=f_nle.copy(), penalized_evidence_trace=trace.copy(),
        support_log_odds_penalty=np.zeros(b, rd), hard_pruning_accepted=np.zeros(b, bool),
        truncation_certified=np.zeros(b, bool),
        active_model_selected=np.full(b, bool(cfg.uamp_polish_prune_tail)),
        active_indices=f_active,
    )
    if exch_acc is not None:
        res["support_repairs_accepted"] = exch_acc
        res["support_exchanges_accepted"] = exch_acc.copy()
    if gcert:  # final diagnostics (4851-4870, 5388-5460)
        tol = rd(cfg.uamp_polish_coordinate_tolerance)
        thr = np.full(b, ratio_threshold_for_evidence_tolerance(cfg.uamp_polish_coordinate_tolerance), rd)
        acert = active_evidence_certificate(mean[rows, f_active], pv[rows, f_active],
                                            f_prior[rows, f_active], f_active)
        stationary = (cert["evidence_gain"] <= tol) & (acert["max_gain"] <= tol)
        in_pen = np.maximum(cert["evidence_gain"], rd(0.0))
        act_pen = np.maximum(acert["max_nondeletion_gain"], np.maximum(acert["max_deletion_gain"], rd(0.0)))
        res.update(
            inactive_max_evidence_ratio=cert["max_ratio"], inactive_best_index=cert["best_index"],
            inactive_evidence_gain=cert["evidence_gain"], inactive_optimal_variance=cert["optimal_variance"],
            active_max_evidence_gain=acert["max_gain"], active_best_index=acert["best_index"],
            active_optimal_variance=acert["optimal_variance"],
            active_max_deletion_gain=acert["max_deletion_gain"],
            coordinate_stationary=stationary, type2_coordinate_stationary=stationary.copy(),
            inactive_ratio_threshold=thr, stationarity_ratio_threshold=thr.copy(),
            inactive_penalized_evidence_gain=in_pen, active_penalized_evidence_gain=act_pen,
            type2_map_coordinate_stationary=(in_pen <= tol) & (act_pen <= tol))
        if cfg.uamp_polish_familywise_error_rate is not None:
            fw = np.full(b, log(max(op.n_grid - k, 1) / cfg.uamp_polish_familywise_error_rate), rd)
            nd = cert["max_ratio"] <= fw
            res.update(familywise_ratio_threshold=fw, familywise_no_discovery=nd,
                       familywise_support_certified=nd.copy())
    return res


def fixed_budget_em_residuals(y, mean, pv, prior, noise, active, prior_floor, op, cfg):
    """solver.py:3408-3496."""
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    b = y.shape[0]
    rows = np.arange(b)[:, None]
    ag = np.maximum(prior[rows, active], tiny)
    ap = pv[rows, active]
    am = mean[rows, active]
    gt = (_abs2(am) + ap + rd(cfg.hyper_rate)) / rd(1.0 + cfg.hyper_shape)
    gt = np.minimum(np.maximum(gt, prior_floor[:, None]), rd(cfg.max_precision))
    gs = np.maximum(np.maximum(np.abs(ag), np.abs(gt)), tiny)
    gres = (np.abs(ag - gt) / gs).max(axis=1)
    if cfg.fixed_noise_variance is not None:
        return gres, np.zeros_like(noise)
    dof = np.clip(rd(1.0) - ap / ag, 0, 1).sum(axis=1, dtype=rd)
    cols = op.fourier_columns(active)
    pred = (cols @ am[:, :, None])[:, :, 0]
    energy = _abs2(y - pred).sum(axis=1, dtype=rd)
    m = op.n_samples
    if cfg.noise_update == "em":
        nt = (energy + noise * dof + rd(cfg.noise_rate)) / rd(m + cfg.noise_shape)
    else:
        nt = (energy + rd(cfg.noise_rate)) / np.maximum(rd(m) - dof + rd(cfg.noise_shape), eps)
    nt = np.minimum(np.maximum(nt, prior_floor), rd(cfg.max_precision))
    ns = np.maximum(np.maximum(np.abs(noise), np.abs(nt)), tiny)
    return gres.astype(rd), (np.abs(noise - nt) / ns).astype(rd)


def fbme_solve(data, grid, profile: str = "stable", *, polish_size: int = 32,
               chol_mode: str = "cuda", observation_mask=None):
    """The FBME-Fast / FBME-Stable plan replay (profiles.py:35-148),
    optionally under an observation mask (sbl_2d, solver.py:986-1024)."""
    cfg = OracleConfig.stable(polish_size) if profile == "stable" else OracleConfig.fastest(polish_size)
    return fast_sbl_uamp(data, grid, cfg, chol_mode=chol_mode, observation_mask=observation_mask)


# ---------------------------------------------------------------------------
# mode="cg": PCG + Hutchinson posterior (solver.py:1194-1221, 1314-1904,
# 2991-3036, 3156-3181, 5582-5848, 6086-6138)
# ---------------------------------------------------------------------------


def cg_probe_count(cfg: OracleConfig, n_grid: int, n_samples: int) -> int:
    """solver.py:1193-1208."""
    maximum = cfg.hutchinson_probes
    if cfg.auto_probe_scaling:
        under = n_grid / n_samples
        rec = 8.0 * under ** 0.5
        if under > 16.0:
            rec = max(rec, 2.0 * under)
        maximum = min(cfg.max_hutchinson_probes, max(cfg.hutchinson_probes, int(rec + 0.999999)))
    return maximum


def cg_schedule(iteration: int, cfg: OracleConfig, maximum_probes: int):
    """solver.py:6086-6118 (probe count, tolerance)."""
    if not cfg.adaptive_cg:
        return maximum_probes, cfg.cg_tolerance
    initial = min(cfg.initial_hutchinson_probes, maximum_probes) if cfg.adaptive_probes else maximum_probes
    if iteration <= 5:
        return initial, max(cfg.cg_initial_tolerance, cfg.cg_tolerance)
    if iteration <= 15:
        mid = (min(maximum_probes, max(initial, min(24, maximum_probes))) if cfg.adaptive_probes
               else maximum_probes)
        return mid, max(cfg.cg_tolerance, (cfg.cg_initial_tolerance * cfg.cg_tolerance) ** 0.5)
    return maximum_probes, cfg.cg_tolerance


def rademacher_probes(batch: int, n_samples: int, count: int, seed: int):
    """solver.py:5979-6000 with torch's CPU generator (the reference's
    stream on CPU).  Returns [B, M, P] complex."""
    import torch

    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    r = 2 * torch.randint(0, 2, (batch, n_samples, count), generator=g) - 1
    return r.numpy().astype(np.float64)


def low_rank_preconditioner(prior, noise, op: PrefixOperator, rank: int, chol_mode: str,
                            jitter_multiplier: float):
    """solver.py:5786-5833."""
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    rank = min(rank, op.n_samples, op.n_grid)
    total = prior.sum(axis=1, dtype=rd)
    if rank == 0:
        return (noise + total).astype(rd), None, None
    idx = _topk_indices(prior, rank)
    vals = np.take_along_axis(prior, idx, axis=1)
    cols = op.fourier_columns(idx)
    factors = (cols * np.sqrt(vals)[:, None, :]).astype(op.cdtype)
    omitted = np.maximum(total - vals.sum(axis=1, dtype=rd), rd(0.0))
    background = np.maximum(noise + omitted, eps * total).astype(rd)
    gram = np.conj(np.swapaxes(factors, 1, 2)) @ factors
    eye = np.eye(rank, dtype=op.cdtype)
    small = eye + gram / background[:, None, None]
    small = rd(0.5) * (small + np.conj(np.swapaxes(small, 1, 2)))
    chol = _stable_cholesky(small, tiny, eps, mode=chol_mode, multiplier=max(10.0, jitter_multiplier),
                            fallback=(10.0, 1e2, 1e3, 1e4, 1e5))
    if chol is None:
        return (noise + total).astype(rd), None, None
    inv = np.linalg.inv(chol)
    small_inv = np.conj(np.swapaxes(inv, 1, 2)) @ inv
    return background, factors, small_inv


def apply_low_rank(value, pre):
    """solver.py:5836-5848."""
    background, factors, small_inv = pre
    base = value / background[:, None, None]
    if factors is None:
        return base
    projected = np.conj(np.swapaxes(factors, 1, 2)) @ value
    w = small_inv @ (projected / background[:, None, None])
    return base - (factors @ w) / background[:, None, None]


def pcg(rhs, prior, noise, op: PrefixOperator, cfg: OracleConfig, *, initial, tolerance,
        chol_mode="cuda", matvec_mode="tbt"):
    """solver.py:5582-5723 with the low-rank preconditioner.  ``matvec``
    "tbt" (the default, solver.py:2995-2999) applies Q through its BTTB
    embedding spectrum (operators.py:299-355); "fourier" applies
    Q v = noise v + A(prior * A^H v) (operators.py:357-371).
    ``fixed_iterations > 0`` keeps the best checkpoint (solver.py:5631-5694)."""
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    fixed_iterations = cfg.cg_fixed_iterations
    if matvec_mode == "tbt":
        spectrum = op.toeplitz_spectrum(prior, noise)

        def matvec(v):
            return op.toeplitz_matvec(v, spectrum)
    else:
        def matvec(v):
            return noise[:, None, None] * v + op.forward(prior[:, :, None] * op.adjoint(v))

    if initial is None:
        x = np.zeros_like(rhs)
        r = rhs.copy()
    else:
        x = initial.copy()
        r = rhs - matvec(x)
    pre = low_rank_preconditioner(prior, noise, op, cfg.cg_preconditioner_rank, chol_mode,
                                  cfg.cuda_cholesky_jitter_multiplier)
    z = apply_low_rank(r, pre)
    d = z.copy()
    rho = np.real((np.conj(r) * z).sum(axis=1))
    init_norm = np.maximum(np.linalg.norm(rhs, axis=1), eps)
    best_x = x.copy() if fixed_iterations > 0 else None
    best_rel = np.linalg.norm(r, axis=1) / init_norm if fixed_iterations > 0 else None
    active = np.linalg.norm(r, axis=1) > tolerance * init_norm
    d = np.where(active[:, None, :], d, 0)
    it = 0
    limit = fixed_iterations if fixed_iterations > 0 else cfg.cg_max_iter
    for it in range(1, limit + 1):
        qd = matvec(d)
        curv = np.real((np.conj(d) * qd).sum(axis=1))
        valid = active & np.isfinite(curv) & np.isfinite(rho) & (curv > tiny) & (rho > tiny)
        alpha = np.where(valid, rho / np.maximum(curv, tiny), 0.0)
        x = x + alpha[:, None, :] * d
        r = r - alpha[:, None, :] * qd
        active = valid
        if it % cfg.cg_check_interval == 0 or it == limit:
            r = rhs - matvec(x)
            rel = np.linalg.norm(r, axis=1) / init_norm
            if fixed_iterations > 0:
                improved = rel < best_rel
                best_x = np.where(improved[:, None, :], x, best_x)
                best_rel = np.minimum(best_rel, rel)
            res_active = np.isfinite(rel) & (rel > tolerance)
            active = active & res_active if fixed_iterations > 0 else res_active
            z = apply_low_rank(r, pre)
            rr = np.real((np.conj(r) * z).sum(axis=1))
            active = active & np.isfinite(rr) & (rr > tiny)
            d = np.where(active[:, None, :], z, 0)
            rho = np.where(active, rr, rho)
            if fixed_iterations == 0 and not active.any():
                break
            continue
        z = apply_low_rank(r, pre)
        new_rho = np.real((np.conj(r) * z).sum(axis=1))
        upd = active & np.isfinite(new_rho) & (new_rho > tiny)
        beta = np.where(upd, new_rho / np.maximum(rho, tiny), 0.0)
        d = z + beta[:, None, :] * d
        d = np.where(upd[:, None, :], d, 0)
        rho = np.where(upd, new_rho, rho)
        active = upd
    out = best_x if best_x is not None else x
    return out.astype(op.cdtype), it


def select_active_indices(prior, minimum_size, maximum_size, tail_fraction):
    """solver.py:3184-3216: the ARD active set of a single scene once at
    most ``maximum_size`` coefficients hold 1 - tail_fraction of the prior
    variance (largest first, ties by index), else None."""
    if prior.shape[0] != 1 or not np.isfinite(prior).all():
        return None
    rd = prior.dtype.type
    maximum = min(maximum_size, prior.shape[1])
    order = np.argsort(-prior[0], kind="stable")[:maximum]
    values = prior[0, order]
    target = rd(1.0 - tail_fraction) * prior.sum(axis=1, dtype=rd)[0]
    if values.sum(dtype=rd) < target:
        return None
    cumulative = np.cumsum(values, dtype=rd)
    required = min(int(np.searchsorted(cumulative, target, side="left")), maximum - 1) + 1
    size = min(maximum, max(minimum_size, required))
    return order[None, :size]


def project_relevance(prior, dd, n_samples, eps):
    """solver.py:3156-3181."""
    rel = np.clip(prior * dd, 0, 1)
    raw = rel.sum(axis=1)
    scale = np.minimum(1.0, n_samples * (1.0 - 10.0 * eps) / np.maximum(raw, eps))
    return rel * scale[:, None]


def lag_index(op: PrefixOperator) -> np.ndarray:
    """operators.py:191-205: flat grid index of the lag m - m' (mod N) of
    every sample pair, [M, M]."""
    c = op.sample_coordinates
    lag = np.remainder(c[:, None, :] - c[None, :, :], np.array(op.grid))
    return lag[..., 0] * op.grid[1] + lag[..., 1]


def dense_posterior(y, prior, noise, op: PrefixOperator, *, chol_mode, chol_multiplier):
    """solver.py:2962-2990 with 3025-3035: the exact posterior through the
    data covariance Q = noise I + A diag(prior) A^H (operators.py:282-297,
    built from the FFT of the prior at the sample lags), its Cholesky
    factor, Q^-1 y and the data diagonal diag(A^H Q^-1 A) from the lag sums
    of Q^-1 (operators.py:418-442).  Returns (mean, posterior variance,
    data diagonal)."""
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    b, n, m = prior.shape[0], op.n_grid, op.n_samples
    li = lag_index(op)
    lags = np.fft.fft2(prior.reshape(b, *op.grid).astype(op.cdtype), axes=(1, 2)).reshape(b, n)
    q = lags[:, li] + noise[:, None, None].astype(op.cdtype) * np.eye(m, dtype=op.cdtype)
    chol = _stable_cholesky(q, tiny, eps, mode=chol_mode, multiplier=chol_multiplier,
                            fallback=(1.0, 10.0, 100.0, 1000.0))
    if chol is None:
        raise RuntimeError("Data covariance is not numerically positive definite.")
    eye = np.broadcast_to(np.eye(m, dtype=op.cdtype), (b, m, m))
    rhs = np.concatenate([y[:, :, None], eye], axis=2)
    fwd = _tri_solve(chol, rhs)
    solved = _tri_solve(np.conj(np.swapaxes(chol, 1, 2)), fwd, upper=True)
    q_inv_y, q_inv = solved[:, :, 0], solved[:, :, 1:]
    lag_sums = np.zeros((b, n), op.cdtype)
    for i in range(b):
        np.add.at(lag_sums[i], li.reshape(-1), q_inv[i].reshape(-1))
    dd = (rd(n) * np.fft.ifft2(lag_sums.reshape(b, *op.grid), axes=(1, 2))).real.reshape(b, n).astype(rd)
    lifted = op.adjoint_flat(q_inv_y.astype(op.cdtype))
    mean = (prior * lifted).astype(op.cdtype)
    pv = np.maximum(prior - np.square(prior) * dd, rd(0.0)).astype(rd)
    return mean, pv, dd


def fast_sbl_dense(data, grid, cfg: OracleConfig, *, chol_mode="cuda"):
    """``fast_sbl`` with ``mode="dense"`` (solver.py:925-2393, posterior
    2962-2990): the cg EM loop with the exact posterior, ``damping`` alone
    and ``min_iter`` as the minimum."""
    return fast_sbl_cg(data, grid, cfg, chol_mode=chol_mode, dense=True)


def fast_sbl_cg(data, grid, cfg: OracleConfig, *, probes=None, chol_mode="cuda", dense=False):
    """``fast_sbl`` with ``mode="cg"``.  A single scene with ``active_set``
    switches to the exact reduced posterior on the selected ARD set once the
    variance tail is small (solver.py:1316-1341, 3184-3216), after which the
    omitted prior variances stay fixed (1684-1693).  ``probes``: [B, M, Pmax]
    (default: the reference's CPU Rademacher stream).  ``dense``: mode="dense"
    (fast_sbl_dense)."""
    data = np.asarray(data)
    cdtype = np.complex128 if data.dtype in (np.complex128, np.float64) else np.complex64
    single = data.ndim == 2
    y3 = data[None] if single else data
    b = y3.shape[0]
    op = PrefixOperator(grid, y3.shape[1:], cdtype)
    rd = op.rdtype
    eps, tiny = _finfo(rd)
    n, m = op.n_grid, op.n_samples
    y = y3.reshape(b, m).astype(cdtype)
    # initialisation: identical to the uamp branch (solver.py:1063-1159)
    dp = np.maximum(_abs2(y).mean(axis=1, dtype=rd), eps).astype(rd)
    floor = np.maximum(dp * rd(cfg.min_variance), tiny).astype(rd)
    uniform = dp[:, None] / rd(n)
    if cfg.initialization == "backprojection":
        bp = op.adjoint_flat(y)
        e = _abs2(bp)
        structured = e / np.maximum(e.sum(axis=1, keepdims=True, dtype=rd), eps) * dp[:, None]
        prior = rd(cfg.initialization_blend) * structured + rd(1 - cfg.initialization_blend) * uniform
    else:
        prior = np.broadcast_to(uniform, (b, n)).copy()
    prior = np.maximum(prior, floor[:, None]).astype(rd)
    noise = (np.full(b, cfg.fixed_noise_variance, rd) if cfg.fixed_noise_variance is not None
             else np.maximum(rd(cfg.initial_noise_fraction) * dp, floor).astype(rd))
    pmax = 0 if dense else cg_probe_count(cfg, n, m)
    if not dense:
        if probes is None:
            probes = rademacher_probes(b, m, pmax, cfg.seed)
        probes = np.asarray(probes).astype(cdtype)
        lifted_probes = op.adjoint(probes)
    minimum = cfg.min_iter if dense else max(cfg.min_iter, cfg.cg_min_iter)
    limit = cfg.max_iter
    conv = cfg.tol > 0.0 and minimum < limit
    keep = rd(cfg.damping if dense else max(cfg.damping, cfg.cg_damping))
    prev_mean = np.zeros((b, n), cdtype)
    solution = None
    streak = 0
    converged = False
    hist = {"relative_change": [], "noise_variance": [], "effective_dof": [], "cg_iterations": [],
            "active_set_size": []}
    active = None
    columns = gram = None

    def reduced():
        """solver.py:3897-3920: the reduced posterior with the omitted
        variance as an isotropic loading."""
        cd = np.conj(np.swapaxes(columns, 1, 2)) @ y[:, :, None]
        mean_a, pv_a, dd_a, _ = active_posterior_with_evidence(
            y, prior, noise, op, active, columns=columns, gram=gram, column_data=cd,
            data_energy=_abs2(y).sum(axis=1, dtype=rd), chol_mode=chol_mode,
            chol_multiplier=cfg.cuda_cholesky_jitter_multiplier, tail_loading=None)
        return mean_a.astype(cdtype), pv_a.astype(rd), dd_a.astype(rd)

    it = 0
    for it in range(1, limit + 1):
        if (not dense and cfg.active_set and b == 1 and active is None and it >= cfg.active_set_start
                and (it - cfg.active_set_start) % cfg.active_set_check_interval == 0):
            active = select_active_indices(prior, cfg.active_set_min_size, cfg.active_set_max_size,
                                           cfg.active_set_tail_fraction)
            if active is not None:
                columns = op.fourier_columns(active).astype(cdtype)
                gram = np.conj(np.swapaxes(columns, 1, 2)) @ columns
                solution = None
        if dense:
            mean, pv, dd = dense_posterior(y, prior, noise, op, chol_mode=chol_mode,
                                           chol_multiplier=cfg.cuda_cholesky_jitter_multiplier)
            cg_it = 0
        else:
            count, tol_cg = cg_schedule(it, cfg, pmax)
            tol_cg = max(tol_cg, 3.0 * float(eps) ** 0.5)
        if active is not None:
            mean, pv, dd = reduced()
            cg_it = 0
        if active is None and not dense:
            rhs = np.concatenate([y[:, :, None], probes[:, :, :count]], axis=2)
            if cfg.cg_warm_start and solution is not None and solution.shape[2] != 1 + count:
                rs = np.zeros((b, m, 1 + count), cdtype)
                sh = min(1 + count, solution.shape[2])
                rs[:, :, :sh] = solution[:, :, :sh]
                solution = rs
            sol, cg_it = pcg(rhs, prior, noise, op, cfg, initial=solution if cfg.cg_warm_start else None,
                             tolerance=tol_cg, chol_mode=chol_mode, matvec_mode=cfg.cg_matvec)
            lifted = op.adjoint(sol)
            dd = np.maximum(np.real(lifted[:, :, 1:] * np.conj(lifted_probes[:, :, :count])).mean(axis=2),
                            0.0).astype(rd)
            mean = (prior * lifted[:, :, 0]).astype(cdtype)
            pv = np.maximum(prior - np.square(prior) * dd, 0.0).astype(rd)
            solution = sol if cfg.cg_warm_start else None
        rel = project_relevance(prior, dd, m, eps).astype(rd)
        dof = rel.sum(axis=1, dtype=rd)
        # MacKay precision update (solver.py:1669-1677)
        prec = (rel + rd(cfg.hyper_shape)) / (_abs2(mean) + rd(cfg.hyper_rate))
        prec = np.clip(prec, rd(1.0 / cfg.max_precision), rd(cfg.max_precision))
        new_prior = (rd(1.0) / prec).astype(rd)
        if active is not None:  # ARD deletion is permanent (solver.py:1684-1693)
            keep_mask = np.zeros((b, n), bool)
            keep_mask[0, active[0]] = True
            new_prior = np.where(keep_mask, new_prior, prior).astype(rd)
        # noise update (solver.py:1737-1768)
        residual = y - op.forward_flat(mean)
        energy = _abs2(residual).sum(axis=1, dtype=rd)
        if cfg.fixed_noise_variance is not None:
            new_noise = np.full(b, cfg.fixed_noise_variance, rd)
        elif cfg.noise_update == "em":
            new_noise = (energy + noise * dof + rd(cfg.noise_rate)) / rd(m + cfg.noise_shape)
        else:
            new_noise = (energy + rd(cfg.noise_rate)) / np.maximum(rd(m) - dof + rd(cfg.noise_shape), eps)
        new_noise = np.maximum(new_noise, floor)
        prior = np.maximum(keep * prior + (rd(1.0) - keep) * new_prior, floor[:, None]).astype(rd)
        noise = (new_noise if cfg.fixed_noise_variance is not None
                 else keep * noise + (rd(1.0) - keep) * new_noise).astype(rd)
        should_check = conv and it >= minimum and ((it - minimum) % cfg.convergence_check_interval == 0
                                                   or it == limit)
        den = np.maximum(np.linalg.norm(mean, axis=1), eps)
        change = float((np.linalg.norm(mean - prev_mean, axis=1) / den).max())
        prev_mean = mean
        hist["relative_change"].append(change)
        hist["noise_variance"].append(float(noise.mean()))
        hist["effective_dof"].append(float(dof.mean()))
        hist["cg_iterations"].append(cg_it)
        hist["active_set_size"].append(0 if active is None else int(active.shape[1]))
        if should_check:
            streak = streak + 1 if change <= cfg.tol else 0
            if streak >= cfg.convergence_patience:
                converged = True
                break
    # final posterior: all probes, or the reduced posterior after a switch
    # (solver.py:2023-2080)
    if dense:
        mean, pv, dd = dense_posterior(y, prior, noise, op, chol_mode=chol_mode,
                                       chol_multiplier=cfg.cuda_cholesky_jitter_multiplier)
    elif active is not None:
        mean, pv, dd = reduced()
    else:
        rhs = np.concatenate([y[:, :, None], probes], axis=2)
        if cfg.cg_warm_start and solution is not None and solution.shape[2] != rhs.shape[2]:
            rs = np.zeros_like(rhs)
            sh = min(rhs.shape[2], solution.shape[2])
            rs[:, :, :sh] = solution[:, :, :sh]
            solution = rs
        sol, _ = pcg(rhs, prior, noise, op, cfg, initial=solution if cfg.cg_warm_start else None,
                     tolerance=max(cfg.cg_tolerance, 3.0 * float(eps) ** 0.5), chol_mode=chol_mode,
                     matvec_mode=cfg.cg_matvec)
        lifted = op.adjoint(sol)
        dd = np.maximum(np.real(lifted[:, :, 1:] * np.conj(lifted_probes)).mean(axis=2), 0.0).astype(rd)
        mean = (prior * lifted[:, :, 0]).astype(cdtype)
        pv = np.maximum(prior - np.square(prior) * dd, 0.0).astype(rd)
    dof = project_relevance(prior, dd, m, eps).sum(axis=1, dtype=rd)
    shape = tuple(grid)
    out = dict(x=mean.reshape((b,) + shape), posterior_variance=pv.reshape((b,) + shape),
               precision=(rd(1.0) / prior).reshape((b,) + shape), noise_variance=noise,
               effective_dof=dof.astype(rd), iterations=it, converged=converged,
               mode="dense" if dense else "cg",
               history=hist, relative_change=hist["relative_change"][-1],
               active_set_size=0 if active is None else int(active.shape[1]),
               active_indices=None if active is None else active[0])
    if single:
        for key in ("x", "posterior_variance", "precision", "noise_variance", "effective_dof"):
            out[key] = out[key][0]
    return out
