"""Eager entry points ``fast_sbl`` / ``sbl_2d`` / ``sbl_1d`` (drop-in for
torch_sbl/solver.py:865-1036).

Mode resolution follows the reference (``auto`` -> ``dense`` when
``M <= dense_threshold`` on CUDA, else ``cg``).  ``mode="uamp"`` runs the
FBME device path (native plan cached by shape and configuration);
``mode="cg"`` runs the PCG + Hutchinson device path.  Inputs must be on a
CUDA device; there is no CPU execution.
"""

from __future__ import annotations

from dataclasses import fields
from math import prod
from typing import Any, Sequence

import torch
from torch import Tensor

from .config import SBLConfig
from .engine import FBMEEngine, check_supported
from .result import SBLResult

_ENGINE_CACHE: dict[tuple, FBMEEngine] = {}
_CACHE_LIMIT = 4


def clear_operator_cache() -> None:
    """Release cached native plans (shape/config keyed), e.g. between jobs."""
    for eng in _ENGINE_CACHE.values():
        eng.close()
    _ENGINE_CACHE.clear()


def _config_key(cfg: SBLConfig) -> tuple:
    return tuple((f.name, str(getattr(cfg, f.name))) for f in fields(cfg))


def _resolve_device(requested: Any, tensor: Tensor) -> torch.device:
    """solver.py:6141-6157."""
    if str(requested) != "auto":
        device = torch.device(requested)
        if device.type == "cuda" and not torch.cuda.is_available():
            raise RuntimeError("CUDA was requested but is not available.")
        if device.type == "cuda" and device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        return device
    if tensor.device.type != "cpu":
        return tensor.device
    if torch.cuda.is_available():
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _engine(batch: int, grid, sample, cfg: SBLConfig, device: torch.device) -> FBMEEngine:
    key = (batch, tuple(grid), tuple(sample), str(device), _config_key(cfg))
    eng = _ENGINE_CACHE.get(key)
    if eng is None:
        if len(_ENGINE_CACHE) >= _CACHE_LIMIT:
            _ENGINE_CACHE.pop(next(iter(_ENGINE_CACHE))).close()
        eng = FBMEEngine(batch, grid, sample, cfg, device)
        _ENGINE_CACHE[key] = eng
    return eng


def fast_sbl(data: Any, grid_shape: Sequence[int], *, config: SBLConfig | None = None,
             observation_mask: Any | None = None) -> SBLResult:
    """Fourier SBL on the B200: ``y = crop(fftn(x)) + noise``, leading
    dimensions are independent scenes."""
    cfg = config or SBLConfig()
    cfg.validate()
    if cfg.learn_snapshot_covariance:
        raise ValueError("learn_snapshot_covariance is available through sbl_2d only.")
    if cfg.phase_error_correction:
        raise ValueError("phase_error_correction is available through sbl_2d only.")
    grid = tuple(int(v) for v in grid_shape)
    if len(grid) not in (1, 2):
        raise ValueError("grid_shape must contain one or two dimensions.")
    if cfg.uamp_support_false_alarm_budget is not None and cfg.uamp_support_false_alarm_budget >= prod(grid):
        raise ValueError(
            "uamp_support_false_alarm_budget must be smaller than the reconstruction grid size.")
    if (cfg.spatial_coupling > 0.0 or cfg.learn_spatial_coupling) and len(grid) != 2:
        raise ValueError("spatial_coupling is only defined for a 2-D grid.")
    tensor = torch.as_tensor(data)
    if tensor.ndim < len(grid):
        raise ValueError("data has fewer dimensions than grid_shape.")
    sample = tuple(int(v) for v in tensor.shape[-len(grid):])
    batch_shape = tuple(int(v) for v in tensor.shape[: -len(grid)])
    if any(m > n for m, n in zip(sample, grid)):
        raise ValueError("Observed dimensions cannot exceed reconstruction dimensions.")
    device = _resolve_device(cfg.device, tensor)
    if device.type != "cuda":
        raise RuntimeError("the FBME B200 path runs on CUDA devices only")
    mask = None
    if observation_mask is not None:  # solver.py:986-1000
        mask = torch.as_tensor(observation_mask, device=device, dtype=torch.bool)
        if tuple(mask.shape) != sample:
            raise ValueError("observation_mask must match the trailing data dimensions.")
        if not bool(mask.any()):
            raise ValueError("observation_mask must retain at least one sample.")
        if cfg.offgrid_refinement:
            raise ValueError("Run off-grid refinement after masked reconstruction.")
    if tensor.dtype in (torch.complex128, torch.float64) or cfg.uamp_polish_high_precision:
        raise NotImplementedError("the B200 path computes in complex64; pass complex64 data")
    n_samples = prod(sample) if mask is None else int(mask.sum())
    threshold = cfg.dense_threshold if device.type == "cuda" else min(cfg.dense_threshold, 512)
    mode = ("dense" if cfg.mode == "auto" and n_samples <= threshold
            else "cg" if cfg.mode == "auto" else cfg.mode)
    if mode == "dense":
        if mask is not None:
            raise NotImplementedError(
                "observation masks run on the B200 uamp path (mode='uamp'); dense mode takes the full block")
        if prod(sample) > 4096:
            raise NotImplementedError("dense mode above 4096 samples is not built on the B200 path")
        from .cg import cg_sbl  # noqa: PLC0415  (the EM loop of the cg plan, exact posterior)
        return cg_sbl(tensor, grid, sample, batch_shape, cfg, device, dense=True)
    if mode == "cg":
        if mask is not None:
            raise NotImplementedError(
                "observation masks run on the B200 uamp path (mode='uamp'); cg mode takes the full block")
        from .cg import cg_sbl  # noqa: PLC0415  (PCG + Hutchinson device path)
        return cg_sbl(tensor, grid, sample, batch_shape, cfg, device)
    check_supported(cfg)
    grid2 = grid if len(grid) == 2 else (1, grid[0])
    sample2 = sample if len(sample) == 2 else (1, sample[0])
    batch = prod(batch_shape) if batch_shape else 1
    y = tensor.to(device=device, dtype=torch.complex64).reshape(batch, -1).contiguous()
    if mask is None:
        eng = _engine(batch, grid2, sample2, cfg, device)
    else:  # a masked plan is built per call (its Gram table depends on the mask)
        eng = FBMEEngine(batch, grid2, sample2, cfg, device, observation_mask=mask.reshape(sample2))
    eng.run(y)
    res = eng.result(batch_shape)
    # eager calls return fresh tensors (the engine's buffers are reused)
    for f in fields(res):
        v = getattr(res, f.name)
        if isinstance(v, Tensor):
            setattr(res, f.name, v.clone())
    if len(grid) == 1:
        for name in ("x", "posterior_variance", "precision", "support_mask"):
            v = getattr(res, name)
            if v is not None:
                setattr(res, name, v.reshape(*batch_shape, grid[0]))
    return res


def sbl_1d(data: Any, grid_size: int, *, config: SBLConfig | None = None,
           observation_mask: Any | None = None) -> SBLResult:
    """1-D spectra ``[..., M]`` -> ``[..., grid_size]`` (solver.py:865-882)."""
    return fast_sbl(data, (int(grid_size),), config=config, observation_mask=observation_mask)


def sbl_2d(data: Any, grid_shape: Sequence[int], *, config: SBLConfig | None = None,
           observation_mask: Any | None = None) -> SBLResult:
    """2-D images ``[..., M1, M2]`` -> ``[..., N1, N2]`` (solver.py:885-922)."""
    shape = tuple(int(v) for v in grid_shape)
    if len(shape) != 2:
        raise ValueError("sbl_2d requires grid_shape=(N1, N2).")
    if config is not None and (config.phase_error_correction or config.learn_snapshot_covariance):
        raise NotImplementedError(
            "autofocus and correlated-MMV reconstruction are outside the B200 FBME path")
    return fast_sbl(data, shape, config=config, observation_mask=observation_mask)
