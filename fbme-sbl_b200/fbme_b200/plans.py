"""Fixed-shape CUDA-Graph plans (drop-in for torch_sbl/cuda_graph.py).

``CUDAGraphSBLPlan`` validates the fixed-budget configuration, builds a
native FBME plan for the example's shape, warms it up on a side stream and
captures one full solve into a ``torch.cuda.CUDAGraph``.  ``replay`` copies
new observations into the plan's input buffer and launches the graph; the
returned ``SBLResult`` tensors are graph-owned and overwritten by the next
replay (torch_sbl/cuda_graph.py:12-124, README "FBME-Fast and FBME-Stable").
"""

from __future__ import annotations

from copy import deepcopy
from math import prod
from typing import Any, Callable, Sequence

import torch
from torch import Tensor

from .config import SBLConfig
from .engine import FBMEEngine, check_supported
from .result import SBLResult


class CUDAGraphSBLPlan:
    """Capture a fixed-shape SBL solve for low-latency replay.

    The input shape, dtype, device, grid, configuration and batch size are
    fixed at construction.  Returned tensors are graph-owned and are
    overwritten by the next replay; clone fields that must outlive it.
    """

    def __init__(self, example_data: Tensor, grid_shape: Sequence[int], *, config: SBLConfig,
                 warmup: int = 3, engine_hook: Callable[[FBMEEngine], None] | None = None,
                 observation_mask: Any | None = None) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA Graph execution requires CUDA.")
        if not isinstance(example_data, Tensor) or not example_data.is_cuda:
            raise ValueError("example_data must be a CUDA tensor.")
        if warmup < 1:
            raise ValueError("warmup must be positive.")
        if config.return_history or config.verbose:
            raise ValueError("CUDA Graph plans require return_history=False and verbose=False.")
        if config.tol > 0.0 or config.eager_change_tracking:
            raise ValueError(
                "CUDA Graph plans require a fixed iteration budget: set tol=0 and "
                "eager_change_tracking=False.")
        if (config.phase_error_correction or config.range_migration_correction
                or config.offgrid_refinement or config.learn_snapshot_covariance):
            raise ValueError(
                "Capture the core SBL stage only; motion, off-grid, and snapshot-covariance "
                "refinement are not graph-static.")
        config.validate()
        if example_data.dtype != torch.complex64:
            raise ValueError("the B200 FBME plans compute in complex64; pass complex64 data.")
        self.grid_shape = tuple(int(v) for v in grid_shape)
        if len(self.grid_shape) != 2:
            raise ValueError("CUDA Graph plans here take a 2-D grid_shape=(N1, N2).")
        if example_data.ndim < 2:
            raise ValueError("data has fewer dimensions than grid_shape.")
        self.config = deepcopy(config)
        self.device = example_data.device
        self.dtype = example_data.dtype
        self.shape = tuple(example_data.shape)
        sample = self.shape[-2:]
        if any(m > n for m, n in zip(sample, self.grid_shape)):
            raise ValueError("Observed dimensions cannot exceed reconstruction dimensions.")
        mode = self.config.mode
        if mode != "uamp":
            raise NotImplementedError(
                "CUDA Graph plans on the B200 path capture mode='uamp' (the FBME profiles).")
        check_supported(self.config)
        self._batch_shape = self.shape[:-2]
        batch = prod(self._batch_shape) if self._batch_shape else 1
        self.input_buffer = torch.empty(self.shape, dtype=self.dtype, device=self.device)
        self.input_buffer.copy_(example_data)
        # observation mask (an extension of the reference's plans, which take
        # the full block; sbl_2d's masked operator, operators.py:57-75)
        self._engine = FBMEEngine(batch, self.grid_shape, sample, self.config, self.device,
                                  observation_mask=observation_mask)
        if engine_hook is not None:  # e.g. the learned warm start, before warm-up and capture
            engine_hook(self._engine)
        flat = self.input_buffer.view(batch, -1)

        warmup_stream = torch.cuda.Stream(device=self.device)
        warmup_stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(warmup_stream):
            for _ in range(warmup):
                self._engine.run(flat)
        torch.cuda.current_stream(self.device).wait_stream(warmup_stream)
        torch.cuda.synchronize(self.device)

        self._graph = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(self._graph):
                self._engine.run(flat)
        except Exception as error:
            raise RuntimeError("CUDA Graph capture failed for this SBL configuration.") from error
        self._result = self._engine.result(self._batch_shape)

    @property
    def result(self) -> SBLResult:
        """Graph-owned output from the most recent replay."""
        return self._result

    def replay(self, data: Tensor | None = None, *, synchronize: bool = False) -> SBLResult:
        """Replay the captured solve, optionally copying a new CUDA input."""
        if data is not None:
            self._validate_input(data)
            self.input_buffer.copy_(data)
        self._graph.replay()
        if synchronize:
            torch.cuda.synchronize(self.device)
        return self._result

    def _validate_input(self, data: Tensor) -> None:
        if not isinstance(data, Tensor) or not data.is_cuda:
            raise ValueError("Replay data must be a CUDA tensor.")
        if data.device != self.device:
            raise ValueError(f"Replay data must be on {self.device}, got {data.device}.")
        if data.dtype != self.dtype:
            raise ValueError(f"Replay data must have dtype {self.dtype}, got {data.dtype}.")
        if tuple(data.shape) != self.shape:
            raise ValueError(f"Replay data must have shape {self.shape}, got {tuple(data.shape)}.")


class RealtimeSBLPlan(CUDAGraphSBLPlan):
    """Low-latency fixed-shape plan for the unified FBME-SBL profile
    (torch_sbl/cuda_graph.py:127-216)."""

    profile = "fbme-sbl-fixed-budget"
    certificate_scope = "fixed-budget-monotone-type2"

    def __init__(self, example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                 warmup: int = 3, config_overrides: dict[str, Any] | None = None,
                 observation_mask: Any | None = None) -> None:
        overrides: dict[str, Any] = {"device": example_data.device, "uamp_polish_size": polish_size}
        if config_overrides is not None:
            overrides.update(config_overrides)
        config = SBLConfig.realtime_hybrid_uamp(**overrides)
        self._validate_realtime_config(config)
        super().__init__(example_data, grid_shape, config=config, warmup=warmup,
                         observation_mask=observation_mask)

    @staticmethod
    def _validate_realtime_config(config: SBLConfig) -> None:
        if not config.uamp_polish_fixed_budget_diagnostics:
            raise ValueError(
                "RealtimeSBLPlan requires fixed-budget diagnostics so the paper objective and "
                "residuals are always reported.")
        if any(v != 0.0 for v in (config.hyper_shape, config.hyper_rate, config.noise_shape,
                                  config.noise_rate)):
            raise ValueError(
                "RealtimeSBLPlan requires zero numerical hyperpriors so its exact evidence gate "
                "matches the stated paper objective.")
        forbidden = {
            "uamp_polish_global_certificate": config.uamp_polish_global_certificate,
            "uamp_polish_support_repairs": config.uamp_polish_support_repairs != 0,
            "uamp_polish_support_growth_steps": config.uamp_polish_support_growth_steps != 0,
            "uamp_polish_support_shrink_steps": config.uamp_polish_support_shrink_steps != 0,
            "uamp_polish_coordinate_steps": config.uamp_polish_coordinate_steps != 0,
            "uamp_polish_noise_coordinate_steps": config.uamp_polish_noise_coordinate_steps != 0,
            "uamp_polish_high_precision": config.uamp_polish_high_precision,
        }
        enabled = [name for name, value in forbidden.items() if value]
        if enabled:
            raise ValueError("RealtimeSBLPlan excludes dynamic research certificates; disable: "
                             + ", ".join(enabled))
        if config.uamp_backend != "triton":
            raise ValueError(
                "RealtimeSBLPlan requires uamp_backend='triton' (the fused device path; on B200 "
                "the sm_100a kernels) so a slow fallback cannot be reported as the real-time path.")


def make_cuda_graph_sbl_plan(example_data: Any, grid_shape: Sequence[int], *,
                             config: SBLConfig | None = None, warmup: int = 3) -> CUDAGraphSBLPlan:
    """Convenience constructor for :class:`CUDAGraphSBLPlan`."""
    tensor = torch.as_tensor(example_data)
    active = config or SBLConfig.fast_hybrid_uamp(device=tensor.device)
    return CUDAGraphSBLPlan(tensor, grid_shape, config=active, warmup=warmup)


def make_realtime_sbl_plan(example_data: Any, grid_shape: Sequence[int], *, polish_size: int = 32,
                           warmup: int = 3,
                           config_overrides: dict[str, Any] | None = None) -> RealtimeSBLPlan:
    """Build the strict fixed-budget real-time CUDA Graph plan."""
    tensor = torch.as_tensor(example_data)
    return RealtimeSBLPlan(tensor, grid_shape, polish_size=polish_size, warmup=warmup,
                           config_overrides=config_overrides)
