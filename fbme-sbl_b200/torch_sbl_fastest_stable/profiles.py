"""Locked FBME-Fast / FBME-Stable CUDA-Graph profiles on B200.

Same constructors, attributes and errors as the reference profiles
(torch_sbl_fastest_stable/profiles.py:22-148 of FBME-SBL v1.1).  Both
profiles share one numerical core and differ in the active-set budget:

    FBME-Fast    2 reduced evaluations, no residual exchange, no diagnostics
    FBME-Stable  3 reduced evaluations, 12-candidate exchange, fixed-budget
                 gamma/noise diagnostics
"""

from __future__ import annotations

from typing import Any, Sequence

import torch
from torch import Tensor

from torch_sbl import PAPER_RELEASE_ID, CUDAGraphSBLPlan, RealtimeSBLPlan, SBLConfig

DUAL_RELEASE_ID = "FBME-SBL-FASTEST-STABLE-v1.0"
CORE_RELEASE_ID = "FBME-SBL-TAES-v1.1"


def _require_frozen_core() -> None:
    if PAPER_RELEASE_ID != CORE_RELEASE_ID:
        raise RuntimeError(
            f"{DUAL_RELEASE_ID} requires core {CORE_RELEASE_ID}, but imported {PAPER_RELEASE_ID}.")


class FastestSBLPlan(CUDAGraphSBLPlan):
    """Minimum-latency locked profile (two exact evaluations, no exchange)."""

    profile = "fbme-sbl-fastest-locked"
    certificate_scope = (
        "exact-evidence-gated-fixed-support;"
        "foreground-fixed-point-diagnostics-disabled"
    )

    def __init__(self, example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                 warmup: int = 3, observation_mask: Any | None = None) -> None:
        _require_frozen_core()
        if example_data.dtype != torch.complex64:
            raise ValueError("FastestSBLPlan is locked to CUDA complex64 arithmetic.")
        config = SBLConfig.paper_hybrid_uamp(
            device=example_data.device,
            uamp_polish_size=polish_size,
            uamp_polish_iterations=2,
            uamp_polish_residual_exchange_size=0,
            uamp_polish_fixed_budget_diagnostics=False,
            uamp_polish_compute_truncation_diagnostic=False,
        )
        if config.uamp_backend != "triton":
            raise RuntimeError("The fastest profile requires the fused device path.")
        super().__init__(example_data, grid_shape, config=config, warmup=warmup,
                         observation_mask=observation_mask)


class StableSBLPlan(RealtimeSBLPlan):
    """Stable locked profile with runtime mathematical diagnostics."""

    profile = "fbme-sbl-stable-locked"
    certificate_scope = "fixed-budget-monotone-type2"

    def __init__(self, example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                 warmup: int = 3, observation_mask: Any | None = None) -> None:
        _require_frozen_core()
        if example_data.dtype != torch.complex64:
            raise ValueError("StableSBLPlan is locked to CUDA complex64 arithmetic.")
        super().__init__(
            example_data, grid_shape, polish_size=polish_size, warmup=warmup,
            observation_mask=observation_mask,
            config_overrides={
                "uamp_polish_iterations": 3,
                "uamp_polish_residual_exchange_size": 12,
                "uamp_polish_fixed_budget_diagnostics": True,
                "uamp_polish_compute_truncation_diagnostic": False,
            },
        )


def make_fastest_plan(example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                      warmup: int = 3, observation_mask: Any | None = None) -> FastestSBLPlan:
    """Build the locked fastest plan (``observation_mask``: B200 extension,
    an [M1, M2] bool mask of observed samples shared by the batch)."""
    return FastestSBLPlan(example_data, grid_shape, polish_size=polish_size, warmup=warmup,
                          observation_mask=observation_mask)


def make_stable_plan(example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                     warmup: int = 3, observation_mask: Any | None = None) -> StableSBLPlan:
    """Build the locked stable plan (``observation_mask`` as for
    make_fastest_plan)."""
    return StableSBLPlan(example_data, grid_shape, polish_size=polish_size, warmup=warmup,
                         observation_mask=observation_mask)
