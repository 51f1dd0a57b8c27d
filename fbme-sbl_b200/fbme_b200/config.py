"""``SBLConfig``: the configuration surface of ``torch_sbl`` (FBME-SBL v1.1).

Same field names, defaults, presets and validation errors as the reference
dataclass (torch_sbl/solver.py:34-717), so existing call sites work
unchanged.  The B200 path reads the hot-path subset (the UAMP/polish and
cg-mode fields); the remaining research fields are accepted and validated
but select paths that are not part of this library (``sbl_2d`` raises
``NotImplementedError`` for them).
"""

from __future__ import annotations

from dataclasses import dataclass, field, fields
from typing import Any

import torch


@dataclass(slots=True)
class SBLConfig:
    """Numerical and iteration settings for fast SBL (solver.py:34-176)."""

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
    cg_matvec: str = "tbt"
    cg_preconditioner: str = "low_rank"
    cg_preconditioner_rank: int = 32
    cg_damping: float = 0.9
    probe_type: str = "rademacher"
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
    cuda_sync_free_cholesky: bool = True
    cuda_cholesky_jitter_multiplier: float = 8.0
    cache_fourier_operator: bool = True
    dense_joint_solve: bool = True
    eager_change_tracking: bool = False
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
    uamp_polish_compute_truncation_diagnostic: bool = True
    uamp_polish_reinitialize: bool = False
    uamp_polish_damping: float = 0.0
    uamp_polish_evidence_gate: bool = False
    uamp_polish_evidence_margin_factor: float = 0.0
    uamp_polish_residual_exchange_size: int = 0
    uamp_polish_max_truncation_delta: float | None = None
    uamp_polish_global_certificate: bool = False
    uamp_polish_support_repairs: int = 0
    uamp_polish_support_growth_steps: int = 0
    uamp_polish_support_shrink_steps: int = 0
    uamp_polish_support_shrink_batch_size: int = 1
    uamp_polish_support_prior: bool = False
    uamp_polish_support_prior_strength: float = 1.0
    uamp_polish_high_precision: bool = False
    uamp_polish_coordinate_steps: int = 0
    uamp_polish_coordinate_tolerance: float = 1e-6
    uamp_polish_coordinate_early_stop: bool = True
    uamp_polish_noise_coordinate_steps: int = 0
    uamp_polish_noise_tolerance: float = 1e-4
    uamp_polish_noise_objective_tolerance: float = 1e-10
    uamp_polish_joint_cycles: int = 1
    uamp_polish_familywise_error_rate: float | None = None
    uamp_polish_fixed_budget_diagnostics: bool = False
    uamp_support_false_alarm_budget: float | None = None
    uamp_backend: str = "auto"
    active_set: bool = True
    active_set_start: int = 30
    active_set_check_interval: int = 2
    active_set_min_size: int = 32
    active_set_max_size: int = 256
    active_set_tail_fraction: float = 5e-2
    joint_sparsity: bool = False
    joint_noise_variance: bool = True
    spatial_coupling: float = 0.0
    spatial_boundary: str = "zero"
    learn_spatial_coupling: bool = False
    spatial_coupling_max: float = 1.0
    spatial_coupling_damping: float = 0.5
    spatial_coupling_steps: int = 4
    spatial_coupling_update_interval: int = 2
    spatial_coupling_penalty: float = 1e-3
    spatial_anisotropy_penalty: float = 1e-2
    learn_snapshot_covariance: bool = False
    snapshot_covariance_model: str = "ar1"
    snapshot_covariance_damping: float = 0.5
    snapshot_covariance_shrinkage: float = 0.05
    snapshot_covariance_floor: float = 1e-3
    snapshot_covariance_start: int = 20
    snapshot_covariance_warmup: int = 20
    snapshot_covariance_min_correlation: float = 0.5
    snapshot_covariance_min_snr_db: float = 10.0
    snapshot_covariance_min_undersampling: float = 48.0
    phase_error_correction: bool = False
    phase_error_axis: int = 1
    phase_basis_rank: int = 6
    phase_optimization_steps: int = 80
    phase_learning_rate: float = 0.05
    phase_smoothness: float = 5.0
    phase_evidence_penalty: float = 1.0
    phase_min_evidence_gain_per_parameter: float = 1.0
    phase_slq_probes: int = 8
    phase_slq_steps: int = 20
    range_dependent_phase: bool = False
    phase_range_basis_rank: int = 2
    range_migration_correction: bool = False
    migration_basis_rank: int = 4
    migration_max_shift: float = 4.0
    migration_smoothness: float = 1.0
    motion_phase_amplitude_penalty: float = 0.2
    motion_migration_amplitude_penalty: float = 0.2
    motion_refinement_steps: int = 40
    motion_refinement_learning_rate: float = 0.02
    offgrid_refinement: bool = False
    offgrid_components: int | None = None
    offgrid_max_components: int = 64
    offgrid_relative_threshold: float = 0.1
    offgrid_minimum_separation: float = 1.5
    offgrid_max_iter: int = 15
    offgrid_tolerance: float = 1e-4
    offgrid_max_step: float = 0.35
    offgrid_damping: float = 1e-3
    offgrid_ridge: float = 1e-7
    seed: int = 0
    device: str | torch.device = "auto"
    return_history: bool = True
    verbose: bool = False
    # B200 extension: how the prefix DFT stages run for mode="uamp".
    # 3 or 6: split-BF16 products on the tensor cores (within 1e-5 relative
    # of the exact operator; FP32 tensor-core accumulation bounds the error).
    # 0: FP32 FFT stages (equal-shape plans, N1 and N2 of the form 2^a or
    # 3 * 2^a up to 512), with the error of an FP32 FFT (~1.5e-7).
    # -1 (default): 0 where that applies, else 3.  cg_dft_terms is the
    # same choice for mode="cg" (3 or 6).
    dft_terms: int = -1
    cg_dft_terms: int = 3

    # ------------------------------------------------------------------ presets
    @classmethod
    def fast_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Low-latency FFT-UAMP preset (solver.py:178-195)."""
        return cls(**{**dict(mode="uamp", tol=0.0, return_history=False,
                             uamp_auto_iterations=True, uamp_polish_size=32,
                             active_set=False), **overrides})

    @classmethod
    def fast_hybrid_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Few-step UAMP + exact active-set EM preset (solver.py:197-227)."""
        base = dict(mode="uamp", max_iter=200, min_iter=1, tol=0.0, return_history=False,
                    uamp_auto_iterations=True, uamp_min_iter=3, uamp_iteration_offset=1.0,
                    uamp_iteration_scale=1.0, uamp_polish_size=32, uamp_polish_iterations=2,
                    uamp_polish_prune_tail=True, uamp_polish_reinitialize=True,
                    uamp_polish_damping=0.0, uamp_polish_evidence_gate=True,
                    uamp_polish_residual_exchange_size=0, active_set=False)
        return cls(**{**base, **overrides})

    @classmethod
    def paper_hybrid_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Unified fixed-budget monotone-evidence preset (solver.py:229-280)."""
        base = dict(device="cuda", uamp_backend="triton", tol=0.0, return_history=False,
                    eager_change_tracking=False, hyper_shape=0.0, hyper_rate=0.0,
                    noise_shape=0.0, noise_rate=0.0, uamp_iteration_offset=0.0,
                    uamp_iteration_scale=0.8, uamp_damping=0.05, uamp_adaptive_damping=False,
                    uamp_polish_iterations=3, uamp_polish_global_certificate=False,
                    uamp_polish_support_repairs=0, uamp_polish_support_growth_steps=0,
                    uamp_polish_support_shrink_steps=0, uamp_polish_support_prior=False,
                    uamp_polish_high_precision=False, uamp_polish_coordinate_steps=0,
                    uamp_polish_noise_coordinate_steps=0,
                    uamp_polish_residual_exchange_size=12,
                    uamp_polish_evidence_margin_factor=64.0,
                    uamp_polish_compute_truncation_diagnostic=False,
                    uamp_polish_familywise_error_rate=None,
                    uamp_polish_fixed_budget_diagnostics=True,
                    uamp_support_false_alarm_budget=0.5, phase_error_correction=False,
                    range_migration_correction=False, offgrid_refinement=False,
                    learn_snapshot_covariance=False)
        return cls.fast_hybrid_uamp(**{**base, **overrides})

    @classmethod
    def realtime_hybrid_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Fixed-budget CUDA-Graph real-time preset (solver.py:282-298)."""
        return cls.paper_hybrid_uamp(**overrides)

    @classmethod
    def certified_hybrid_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Hybrid preset with exact Type-II coordinate diagnostics (solver.py:300-316)."""
        return cls.fast_hybrid_uamp(**{**dict(uamp_polish_global_certificate=True,
                                              uamp_polish_iterations=4,
                                              uamp_polish_support_repairs=1), **overrides})

    @classmethod
    def taes_hybrid_uamp(cls, **overrides: Any) -> "SBLConfig":
        """Evidence-monotone Type-II research preset (solver.py:318-350)."""
        base = dict(uamp_polish_global_certificate=True, uamp_polish_iterations=8,
                    uamp_polish_support_repairs=1, uamp_polish_support_growth_steps=64,
                    uamp_polish_support_shrink_steps=64, uamp_polish_support_shrink_batch_size=8,
                    uamp_polish_support_prior=True, uamp_polish_support_prior_strength=1.0,
                    uamp_polish_high_precision=True, uamp_polish_coordinate_steps=64,
                    uamp_polish_coordinate_tolerance=1e-3, uamp_polish_noise_coordinate_steps=16,
                    uamp_polish_noise_tolerance=1e-4, uamp_polish_noise_objective_tolerance=1e-10,
                    uamp_polish_joint_cycles=8, uamp_polish_familywise_error_rate=0.05)
        return cls.fast_hybrid_uamp(**{**base, **overrides})

    # --------------------------------------------------------------- validation
    def validate(self) -> None:
        """Raise ``ValueError`` on the conditions solver.py:352-717 rejects."""
        for message, bad in _rules(self):
            if bad:
                raise ValueError(message)

    def replace(self, **changes: Any) -> "SBLConfig":
        values = {f.name: getattr(self, f.name) for f in fields(self)}
        values.update(changes)
        return SBLConfig(**values)


def _rules(c: SBLConfig):
    """(message, violated) pairs, in the order the reference checks them."""
    gcert = c.uamp_polish_global_certificate
    yield "Iteration counts must be positive.", c.max_iter < 1 or c.min_iter < 1
    yield "damping must satisfy 0 <= damping < 1.", not 0.0 <= c.damping < 1.0
    yield "mode must be 'auto', 'dense', 'cg', or 'uamp'.", c.mode not in ("auto", "dense", "cg", "uamp")
    yield "noise_update must be 'em' or 'evidence'.", c.noise_update not in ("em", "evidence")
    yield ("initialization must be 'uniform' or 'backprojection'.",
           c.initialization not in ("uniform", "backprojection"))
    yield "initialization_blend must be between 0 and 1.", not 0.0 <= c.initialization_blend <= 1.0
    yield ("fixed_noise_variance must be positive.",
           c.fixed_noise_variance is not None and c.fixed_noise_variance <= 0)
    yield "hutchinson_probes must be positive.", c.hutchinson_probes < 1
    yield "initial_hutchinson_probes must be positive.", c.initial_hutchinson_probes < 1
    yield ("max_hutchinson_probes must be >= hutchinson_probes.",
           c.max_hutchinson_probes < c.hutchinson_probes)
    yield "CG tolerances must be positive.", c.cg_tolerance <= 0.0 or c.cg_initial_tolerance <= 0.0
    yield ("convergence check intervals must be positive.",
           c.cg_check_interval < 1 or c.convergence_check_interval < 1)
    yield "cg_fixed_iterations cannot be negative.", c.cg_fixed_iterations < 0
    yield "cg_fixed_iterations cannot exceed cg_max_iter.", c.cg_fixed_iterations > c.cg_max_iter
    yield ("CG minimum iterations and patience must be positive.",
           c.cg_min_iter < 1 or c.convergence_patience < 1)
    yield ("cuda_cholesky_jitter_multiplier must be positive.",
           c.cuda_cholesky_jitter_multiplier <= 0.0)
    yield "cg_matvec must be 'tbt' or 'fourier'.", c.cg_matvec not in ("tbt", "fourier")
    yield ("cg_preconditioner must be 'circulant', 'low_rank', 'nystrom', or 'none'.",
           c.cg_preconditioner not in ("circulant", "low_rank", "nystrom", "none"))
    yield "cg_preconditioner_rank cannot be negative.", c.cg_preconditioner_rank < 0
    yield "cg_damping must satisfy 0 <= cg_damping < 1.", not 0.0 <= c.cg_damping < 1.0
    yield "uamp_damping must satisfy 0 <= uamp_damping < 1.", not 0.0 <= c.uamp_damping < 1.0
    yield "uamp_max_damping must be in [uamp_damping, 1).", not c.uamp_damping <= c.uamp_max_damping < 1.0
    yield "uamp_min_iter must be positive.", c.uamp_min_iter < 1
    yield "uamp_iteration_offset cannot be negative.", c.uamp_iteration_offset < 0.0
    yield "uamp_iteration_scale must be positive.", c.uamp_iteration_scale <= 0.0
    yield "uamp_polish_size cannot be negative.", c.uamp_polish_size < 0
    yield "uamp_polish_iterations must be positive.", c.uamp_polish_iterations < 1
    yield ("uamp_polish_residual_exchange_size must be in [0, 32].",
           not 0 <= c.uamp_polish_residual_exchange_size <= 32)
    yield ("Residual support exchange requires at least two polish evaluations, zero-tail "
           "pruning, and the exact evidence gate.",
           c.uamp_polish_residual_exchange_size > 0 and (
               c.uamp_polish_iterations < 2 or not c.uamp_polish_prune_tail
               or not c.uamp_polish_evidence_gate))
    yield "uamp_polish_damping must satisfy 0 <= damping < 1.", not 0.0 <= c.uamp_polish_damping < 1.0
    yield ("uamp_polish_evidence_margin_factor cannot be negative.",
           c.uamp_polish_evidence_margin_factor < 0.0)
    yield ("uamp_polish_max_truncation_delta must be positive.",
           c.uamp_polish_max_truncation_delta is not None and c.uamp_polish_max_truncation_delta <= 0.0)
    yield ("uamp_polish_support_repairs must be between 0 and 4.",
           not 0 <= c.uamp_polish_support_repairs <= 4)
    yield ("uamp_polish_support_repairs requires uamp_polish_global_certificate=True.",
           c.uamp_polish_support_repairs > 0 and not gcert)
    yield ("uamp_polish_support_growth_steps must be between 0 and 64.",
           not 0 <= c.uamp_polish_support_growth_steps <= 64)
    yield ("uamp_polish_support_growth_steps requires uamp_polish_global_certificate=True.",
           c.uamp_polish_support_growth_steps > 0 and not gcert)
    yield ("uamp_polish_support_shrink_steps must be between 0 and 64.",
           not 0 <= c.uamp_polish_support_shrink_steps <= 64)
    yield ("uamp_polish_support_shrink_steps requires uamp_polish_global_certificate=True.",
           c.uamp_polish_support_shrink_steps > 0 and not gcert)
    yield ("uamp_polish_support_shrink_batch_size must be in [1, 32].",
           not 1 <= c.uamp_polish_support_shrink_batch_size <= 32)
    yield ("uamp_polish_support_prior_strength cannot be negative.",
           c.uamp_polish_support_prior_strength < 0.0)
    yield ("uamp_polish_support_prior requires uamp_polish_global_certificate=True.",
           c.uamp_polish_support_prior and not gcert)
    yield ("uamp_polish_coordinate_steps must be between 0 and 64.",
           not 0 <= c.uamp_polish_coordinate_steps <= 64)
    yield ("uamp_polish_coordinate_tolerance cannot be negative.",
           c.uamp_polish_coordinate_tolerance < 0.0)
    yield ("uamp_polish_coordinate_steps requires uamp_polish_global_certificate=True.",
           c.uamp_polish_coordinate_steps > 0 and not gcert)
    yield ("uamp_polish_noise_coordinate_steps must be between 0 and 64.",
           not 0 <= c.uamp_polish_noise_coordinate_steps <= 64)
    yield "uamp_polish_noise_tolerance must be positive.", c.uamp_polish_noise_tolerance <= 0.0
    yield ("uamp_polish_noise_objective_tolerance cannot be negative.",
           c.uamp_polish_noise_objective_tolerance < 0.0)
    yield ("uamp_polish_joint_cycles must be between 1 and 32.",
           not 1 <= c.uamp_polish_joint_cycles <= 32)
    yield ("uamp_polish_noise_coordinate_steps requires uamp_polish_global_certificate=True.",
           c.uamp_polish_noise_coordinate_steps > 0 and not gcert)
    yield ("Noise-coordinate refinement is incompatible with fixed_noise_variance; either "
           "estimate noise or fix it.",
           c.uamp_polish_noise_coordinate_steps > 0 and c.fixed_noise_variance is not None)
    yield ("uamp_polish_familywise_error_rate must be in (0, 1).",
           c.uamp_polish_familywise_error_rate is not None
           and not 0.0 < c.uamp_polish_familywise_error_rate < 1.0)
    yield ("uamp_polish_familywise_error_rate requires uamp_polish_global_certificate=True.",
           c.uamp_polish_familywise_error_rate is not None and not gcert)
    yield ("Exact Type-II coordinate diagnostics require uamp_polish_prune_tail=True so inactive "
           "variances define the zero-tail active model.",
           gcert and not c.uamp_polish_prune_tail)
    yield ("uamp_polish_fixed_budget_diagnostics requires uamp_polish_prune_tail=True and "
           "uamp_polish_evidence_gate=True.",
           c.uamp_polish_fixed_budget_diagnostics and (
               not c.uamp_polish_prune_tail or not c.uamp_polish_evidence_gate))
    yield ("uamp_support_false_alarm_budget must be positive.",
           c.uamp_support_false_alarm_budget is not None and c.uamp_support_false_alarm_budget <= 0.0)
    yield "uamp_backend must be 'auto', 'torch', or 'triton'.", c.uamp_backend not in ("auto", "torch", "triton")
    yield ("uamp_polish_high_precision=True requires the Torch backend: Triton UAMP currently "
           "supports complex64 only. Use uamp_backend='torch' (or 'auto') for the research path, "
           "or disable high precision for the latency path.",
           c.uamp_polish_high_precision and c.uamp_backend == "triton")
    yield "probe_type must be 'rademacher' or 'hadamard'.", c.probe_type not in ("rademacher", "hadamard")
    yield ("Active-set iteration counts must be positive.",
           c.active_set_start < 1 or c.active_set_check_interval < 1)
    yield "active_set_min_size must be positive.", c.active_set_min_size < 1
    yield "active_set_max_size must be >= active_set_min_size.", c.active_set_max_size < c.active_set_min_size
    yield "active_set_tail_fraction must be in (0, 1).", not 0.0 < c.active_set_tail_fraction < 1.0
    yield "spatial_coupling must be in [0, 1].", not 0.0 <= c.spatial_coupling <= 1.0
    yield "spatial_boundary must be 'zero' or 'circular'.", c.spatial_boundary not in ("zero", "circular")
    yield "spatial_coupling_max must be in (0, 2].", not 0.0 < c.spatial_coupling_max <= 2.0
    yield "spatial_coupling_damping must be in [0, 1).", not 0.0 <= c.spatial_coupling_damping < 1.0
    yield ("Spatial coupling steps and update interval must be positive.",
           c.spatial_coupling_steps < 1 or c.spatial_coupling_update_interval < 1)
    yield ("Spatial coupling penalties cannot be negative.",
           c.spatial_coupling_penalty < 0.0 or c.spatial_anisotropy_penalty < 0.0)
    yield "snapshot_covariance_damping must be in [0, 1).", not 0.0 <= c.snapshot_covariance_damping < 1.0
    yield "snapshot_covariance_shrinkage must be in [0, 1).", not 0.0 <= c.snapshot_covariance_shrinkage < 1.0
    yield "snapshot_covariance_floor must be in (0, 1).", not 0.0 < c.snapshot_covariance_floor < 1.0
    yield "snapshot_covariance_model must be 'ar1' or 'full'.", c.snapshot_covariance_model not in ("ar1", "full")
    yield ("Snapshot-covariance start must be nonnegative and warmup must be positive.",
           c.snapshot_covariance_start < 0 or c.snapshot_covariance_warmup < 1)
    yield ("snapshot_covariance_min_correlation must be in [0, 1).",
           not 0.0 <= c.snapshot_covariance_min_correlation < 1.0)
    yield ("snapshot_covariance_min_undersampling must be at least one.",
           c.snapshot_covariance_min_undersampling < 1.0)
    yield "phase_error_axis must be 0 or 1.", c.phase_error_axis not in (0, 1)
    yield ("Phase basis rank and optimization steps must be positive.",
           c.phase_basis_rank < 1 or c.phase_optimization_steps < 1)
    yield ("Phase optimization settings are invalid.",
           c.phase_learning_rate <= 0.0 or c.phase_smoothness < 0.0)
    yield "phase_evidence_penalty cannot be negative.", c.phase_evidence_penalty < 0.0
    yield ("phase_min_evidence_gain_per_parameter cannot be negative.",
           c.phase_min_evidence_gain_per_parameter < 0.0)
    yield "SLQ requires positive probes and at least 2 steps.", c.phase_slq_probes < 1 or c.phase_slq_steps < 2
    yield "phase_range_basis_rank must be positive.", c.phase_range_basis_rank < 1
    yield "migration_basis_rank must be positive.", c.migration_basis_rank < 1
    yield "Range-migration settings are invalid.", c.migration_max_shift <= 0.0 or c.migration_smoothness < 0.0
    yield ("Motion-amplitude penalties cannot be negative.",
           c.motion_phase_amplitude_penalty < 0.0 or c.motion_migration_amplitude_penalty < 0.0)
    yield ("Motion-refinement settings are invalid.",
           c.motion_refinement_steps < 0 or c.motion_refinement_learning_rate <= 0.0)
    yield "offgrid_components must be positive.", c.offgrid_components is not None and c.offgrid_components < 1
    yield "offgrid_max_components must be positive.", c.offgrid_max_components < 1
    yield "offgrid_relative_threshold must be in (0, 1).", not 0.0 < c.offgrid_relative_threshold < 1.0
    yield "offgrid_minimum_separation cannot be negative.", c.offgrid_minimum_separation < 0.0
    yield ("Off-grid refinement settings are invalid.",
           c.offgrid_max_iter < 1 or c.offgrid_tolerance <= 0.0 or c.offgrid_max_step <= 0.0
           or c.offgrid_damping <= 0.0 or c.offgrid_ridge < 0.0)
    yield "dft_terms must be -1 (automatic), 0 (FP32 FFT), 3 or 6.", c.dft_terms not in (-1, 0, 3, 6)
    yield "cg_dft_terms must be 3 or 6.", c.cg_dft_terms not in (3, 6)


def fbme_profile_config(profile: str = "stable", polish_size: int = 32,
                        sweeps: int | None = None) -> SBLConfig:
    """The configuration of the FBME plans (torch_sbl_fastest_stable/
    profiles.py:63-70 for "fast", 110-115 for "stable"), optionally with a
    fixed UAMP sweep budget instead of the auto rule."""
    if profile not in ("stable", "fast"):
        raise ValueError("profile must be 'stable' or 'fast'")
    over: dict[str, Any] = dict(uamp_polish_size=polish_size,
                                uamp_polish_compute_truncation_diagnostic=False)
    if profile == "stable":
        over.update(uamp_polish_iterations=3, uamp_polish_residual_exchange_size=12,
                    uamp_polish_fixed_budget_diagnostics=True)
    else:
        over.update(uamp_polish_iterations=2, uamp_polish_residual_exchange_size=0,
                    uamp_polish_fixed_budget_diagnostics=False)
    if sweeps is not None:
        over.update(uamp_auto_iterations=False, max_iter=int(sweeps), min_iter=1, uamp_min_iter=1)
    return SBLConfig.paper_hybrid_uamp(**over)
