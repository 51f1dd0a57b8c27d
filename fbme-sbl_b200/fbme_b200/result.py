"""``SBLResult``: the reconstruction and posterior-state container.

Same fields and defaults as the reference dataclass
(torch_sbl/solver.py:720-792), so code that reads a plan's or ``sbl_2d``'s
result works unchanged.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

from torch import Tensor


@dataclass(slots=True)
class SBLResult:
    """Reconstruction and final posterior state."""

    x: Tensor
    posterior_variance: Tensor
    precision: Tensor
    noise_variance: Tensor
    effective_dof: Tensor
    iterations: int
    converged: bool
    relative_change: float
    mode: str
    arithmetic_dtype: str = ""
    uamp_backend_used: str | None = None
    active_set_size: int = 0
    offgrid: Any | None = None
    snapshot_covariance: Tensor | None = None
    snapshot_covariance_active: bool | None = None
    snapshot_snr_db: float | None = None
    learned_spatial_coupling: Tensor | None = None
    phase_error: Tensor | None = None
    phase_candidate: Tensor | None = None
    phase_correction_accepted: bool | None = None
    phase_evidence_gain: float | None = None
    range_migration: Tensor | None = None
    range_migration_candidate: Tensor | None = None
    negative_log_evidence: Tensor | None = None
    evidence_trace: Tensor | None = None
    truncation_delta_bound: Tensor | None = None
    hard_pruning_accepted: Tensor | None = None
    truncation_certified: Tensor | None = None
    inactive_max_evidence_ratio: Tensor | None = None
    inactive_best_index: Tensor | None = None
    inactive_evidence_gain: Tensor | None = None
    inactive_optimal_variance: Tensor | None = None
    support_repairs_accepted: Tensor | None = None
    support_exchanges_accepted: Tensor | None = None
    support_growth_accepted: Tensor | None = None
    support_shrink_accepted: Tensor | None = None
    active_max_evidence_gain: Tensor | None = None
    active_best_index: Tensor | None = None
    active_optimal_variance: Tensor | None = None
    active_max_deletion_gain: Tensor | None = None
    coordinate_steps_accepted: Tensor | None = None
    coordinate_stationary: Tensor | None = None
    inactive_ratio_threshold: Tensor | None = None
    familywise_support_certified: Tensor | None = None
    type2_coordinate_stationary: Tensor | None = None
    stationarity_ratio_threshold: Tensor | None = None
    familywise_ratio_threshold: Tensor | None = None
    familywise_no_discovery: Tensor | None = None
    active_model_selected: Tensor | None = None
    support_log_odds_penalty: Tensor | None = None
    penalized_negative_log_evidence: Tensor | None = None
    penalized_evidence_trace: Tensor | None = None
    inactive_penalized_evidence_gain: Tensor | None = None
    active_penalized_evidence_gain: Tensor | None = None
    type2_map_coordinate_stationary: Tensor | None = None
    noise_coordinate_steps_accepted: Tensor | None = None
    noise_evidence_gradient: Tensor | None = None
    noise_fixed_point_residual: Tensor | None = None
    noise_evidence_gain: Tensor | None = None
    noise_coordinate_stationary: Tensor | None = None
    joint_map_coordinate_stationary: Tensor | None = None
    joint_coordinate_cycles: Tensor | None = None
    fixed_budget_gamma_residual: Tensor | None = None
    fixed_budget_noise_residual: Tensor | None = None
    fixed_budget_objective_decrease: Tensor | None = None
    fixed_budget_monotone: Tensor | None = None
    support_mask: Tensor | None = None
    support_score_threshold: Tensor | None = None
    history: dict[str, list[float]] = field(default_factory=dict)
    # B200 extension: per-scene status bits (0 = ok), see include/fbme_b200.h.
    status: Tensor | None = None
