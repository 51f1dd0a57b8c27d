"""``mode="cg"`` on the B200: PCG + Hutchinson SBL through the native cg plan.

Drop-in for the reference's ``fast_sbl`` / ``sbl_2d`` with ``mode="cg"``
(torch_sbl/solver.py:925-2393).  The host resolves the probe budget
(solver.py:1191-1208) and draws the probes exactly as the reference does
(``_make_probes``, solver.py:5979-6083: a seeded ``torch.Generator`` on the
solve's device), then one native call runs the whole EM loop: prior and
noise initialisation, the PCG solves with the low-rank preconditioner, the
Hutchinson diagonal, the MacKay and noise updates, the convergence test and
the final posterior.

A single scene with ``active_set`` switches to the exact reduced posterior
on its ARD set once the variance tail is small (solver.py:1316-1341): the
native plan selects the set on the device and reads only its size.

Not built here (``NotImplementedError``): joint sparsity, spatial coupling,
the circulant / Nystrom / no preconditioner, off-grid refinement, and active
sets above 1024 coefficients (``active_set_max_size``).
"""

from __future__ import annotations

import ctypes
from math import prod
from typing import Sequence

import numpy as np
import torch
from torch import Tensor

from . import _native as nat
from .config import SBLConfig
from .result import SBLResult


def probe_count(cfg: SBLConfig, n_grid: int, n_samples: int) -> int:
    """Maximum Hutchinson probes (solver.py:1193-1208)."""
    maximum = cfg.hutchinson_probes
    if cfg.auto_probe_scaling:
        under = n_grid / n_samples
        rec = 8.0 * under ** 0.5
        if under > 16.0:
            rec = max(rec, 2.0 * under)
        maximum = min(cfg.max_hutchinson_probes, max(cfg.hutchinson_probes, int(rec + 0.999999)))
    return maximum


def make_probes(batch: int, n_samples: int, count: int, *, device: torch.device, seed: int,
                probe_type: str = "rademacher",
                sample_shape: Sequence[int] | None = None) -> Tensor:
    """Real +-1 probes ``[batch, n_samples, count]`` drawn from the same
    generator stream as the reference (solver.py:5979-6083)."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    if probe_type == "rademacher":
        return (2 * torch.randint(0, 2, (batch, n_samples, count), device=device, generator=gen)
                - 1).to(torch.float32)
    # Hierarchical probing: one Rademacher diagonal per block of Hadamard
    # columns (Gray-code order), rows numbered by interleaving the bits of
    # the sample coordinates so that nearby samples get nearby codes.
    shape = tuple(int(v) for v in (sample_shape or (n_samples,)))
    if prod(shape) != n_samples:
        raise ValueError("probe_shape must have product n_grid.")
    bits = [max(0, (length - 1).bit_length()) for length in shape]
    embedding = 1 << sum(bits)
    if count > embedding:
        raise ValueError("Hadamard probe count cannot exceed its embedding.")
    block = count if count == embedding else min(8, 1 << max(0, count.bit_length() - 1))
    nblocks = (count + block - 1) // block
    signs = 2 * torch.randint(0, 2, (batch, n_samples, nblocks), device=device, generator=gen) - 1
    coords = torch.meshgrid(*[torch.arange(n, device=device) for n in shape], indexing="ij")
    coords = [c.reshape(-1) for c in coords]
    code = torch.zeros(n_samples, dtype=torch.long, device=device)
    out_bit = 0
    for ib in range(max(bits, default=0)):
        for c, nb in zip(coords, bits):
            if ib < nb:
                code |= ((c >> ib) & 1) << out_bit
                out_bit += 1
    col = torch.arange(count, device=device) % block
    col = col ^ (col >> 1)
    anded = code[:, None] & col[None, :]
    parity = torch.zeros_like(anded)
    sh = 0
    while (1 << sh) < embedding:
        parity ^= (anded >> sh) & 1
        sh += 1
    hadamard = (1 - 2 * parity).to(torch.float32)
    owner = torch.div(torch.arange(count, device=device), block, rounding_mode="floor")
    return signs.index_select(2, owner).to(torch.float32) * hadamard.unsqueeze(0)


def check_cg_supported(cfg: SBLConfig, batch: int, dense: bool = False) -> None:
    unsupported = {
        "joint_sparsity": cfg.joint_sparsity,
        "spatial_coupling": cfg.spatial_coupling > 0.0 or cfg.learn_spatial_coupling,
        f"cg_preconditioner={cfg.cg_preconditioner!r}": cfg.cg_preconditioner != "low_rank" and not dense,
        "offgrid_refinement": cfg.offgrid_refinement,
    }
    bad = [k for k, v in unsupported.items() if v]
    if bad:
        raise NotImplementedError("the B200 cg path does not implement: " + ", ".join(bad))
    if cfg.active_set and batch == 1 and cfg.active_set_max_size > 1024:
        raise NotImplementedError("active_set_max_size above 1024 is not built on the B200 cg path")
    if cfg.cg_preconditioner_rank > 32:
        raise NotImplementedError("cg_preconditioner_rank above 32 is not built")


def resolve_cg_config(cfg: SBLConfig, n_grid: int, n_samples: int, batch: int = 1,
                      dense: bool = False) -> nat.FbmeCgConfig:
    """Map ``cfg`` to ``FbmeCgConfig``; the active-set switch applies to a
    single scene only (solver.py:1316-1323).  ``dense``: mode="dense", the
    exact posterior through the data covariance (no probes)."""
    c = nat.FbmeCgConfig()
    c.max_iter = cfg.max_iter
    c.min_iter = cfg.min_iter
    c.cg_min_iter = cfg.cg_min_iter
    c.tol = cfg.tol
    c.convergence_patience = cfg.convergence_patience
    c.convergence_check_interval = cfg.convergence_check_interval
    c.hyper_shape = cfg.hyper_shape
    c.hyper_rate = cfg.hyper_rate
    c.noise_shape = cfg.noise_shape
    c.noise_rate = cfg.noise_rate
    c.initial_noise_fraction = cfg.initial_noise_fraction
    c.initialization_blend = (cfg.initialization_blend if cfg.initialization == "backprojection"
                              else -1.0)
    c.fixed_noise_variance = cfg.fixed_noise_variance if cfg.fixed_noise_variance is not None else 0.0
    c.noise_update = 1 if cfg.noise_update == "evidence" else 0
    c.damping = cfg.damping
    c.cg_damping = cfg.cg_damping
    c.min_variance = cfg.min_variance
    c.max_precision = cfg.max_precision
    c.cg_tolerance = cfg.cg_tolerance
    c.cg_initial_tolerance = cfg.cg_initial_tolerance
    c.cg_max_iter = cfg.cg_max_iter
    c.cg_check_interval = cfg.cg_check_interval
    c.cg_fixed_iterations = cfg.cg_fixed_iterations
    c.preconditioner_rank = cfg.cg_preconditioner_rank
    c.probes = probe_count(cfg, n_grid, n_samples)
    c.initial_probes = cfg.initial_hutchinson_probes
    c.adaptive_cg = int(cfg.adaptive_cg)
    c.adaptive_probes = int(cfg.adaptive_probes)
    c.warm_start = int(cfg.cg_warm_start)
    c.jitter_multiplier = cfg.cuda_cholesky_jitter_multiplier
    c.dft_terms = cfg.cg_dft_terms
    switch = cfg.active_set and batch == 1 and not cfg.joint_sparsity and not dense
    c.active_set_start = cfg.active_set_start if switch else 0
    c.active_set_check_interval = cfg.active_set_check_interval
    c.active_set_min_size = cfg.active_set_min_size
    c.active_set_max_size = cfg.active_set_max_size
    c.active_set_tail_fraction = cfg.active_set_tail_fraction
    c.dense = int(dense)
    if dense:
        c.probes = 0
    return c


class CGEngine:
    """A native cg plan for ``batch`` scenes of one shape and configuration."""

    def __init__(self, batch: int, grid: Sequence[int], sample: Sequence[int], cfg: SBLConfig,
                 device: torch.device, dense: bool = False) -> None:
        self.lib = nat.lib()
        if device.type != "cuda":
            raise RuntimeError("the B200 cg path needs a CUDA device")
        self.dense = bool(dense)
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.batch = int(batch)
        self.grid = tuple(int(v) for v in grid)
        self.sample = tuple(int(v) for v in sample)
        self.cfg = cfg
        self.n_grid, self.n_samples = prod(self.grid), prod(self.sample)
        self.native_cfg = resolve_cg_config(cfg, self.n_grid, self.n_samples, self.batch, self.dense)
        self.probes = int(self.native_cfg.probes)
        self._shape = nat.FbmeShape(self.grid[0], self.grid[1], self.sample[0], self.sample[1])
        nbytes = self.lib.fbme_cg_workspace_bytes(ctypes.byref(self._shape), self.batch,
                                                  ctypes.byref(self.native_cfg))
        if nbytes == 0:
            msg = nat.last_error()
            nat.check(nat.FBME_ERR_UNSUPPORTED if ("not built" in msg or "more than" in msg)
                      else nat.FBME_ERR_INVALID, "fbme_cg_workspace_bytes")
        self.workspace = torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=device)
        self._ws_ptr = (self.workspace.data_ptr() + 255) & ~255
        self._plan = ctypes.c_void_p()
        with torch.cuda.device(device):
            rc = self.lib.fbme_cg_create(ctypes.byref(self._shape), self.batch,
                                         ctypes.byref(self.native_cfg), ctypes.c_void_p(self._ws_ptr),
                                         ctypes.c_size_t(nbytes), ctypes.c_void_p(self._stream()),
                                         ctypes.byref(self._plan))
        nat.check(rc, "fbme_cg_create")

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None and self._plan.value:
            torch.cuda.synchronize(self.device)
            self.lib.fbme_cg_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------
    def default_probes(self) -> Tensor:
        """The reference's probes for this solve, as ``[B, P, M]`` floats."""
        cfg = self.cfg
        z = make_probes(self.batch, self.n_samples, self.probes, device=self.device, seed=cfg.seed,
                        probe_type=cfg.probe_type, sample_shape=self.sample)
        return z.permute(0, 2, 1).contiguous()

    def solve(self, y: Tensor, probes: Tensor | None = None) -> SBLResult:
        """``y``: complex64 ``[B, M]``; ``probes``: float ``[B, P, M]`` (default:
        the reference's generator stream)."""
        B, N, M = self.batch, self.n_grid, self.n_samples
        y = y.to(device=self.device, dtype=torch.complex64).reshape(B, M).contiguous()
        if self.dense:  # no probes: a placeholder pointer for the C ABI
            probes = torch.zeros(1, dtype=torch.float32, device=self.device)
        else:
            if probes is None:
                probes = self.default_probes()
            probes = probes.to(device=self.device, dtype=torch.float32).contiguous()
            if tuple(probes.shape) != (B, self.probes, M):
                raise ValueError(f"probes must have shape {(B, self.probes, M)}")
        f32 = dict(dtype=torch.float32, device=self.device)
        x = torch.empty(B, N, dtype=torch.complex64, device=self.device)
        pv = torch.empty(B, N, **f32)
        prec = torch.empty(B, N, **f32)
        noise = torch.empty(B, **f32)
        dof = torch.empty(B, **f32)
        status = torch.zeros(B, dtype=torch.int32, device=self.device)
        budget = self.cfg.uamp_support_false_alarm_budget
        mask = torch.empty(B, N, dtype=torch.bool, device=self.device) if budget is not None else None
        out = nat.FbmeCgOutputs()
        out.x, out.posterior_variance, out.precision = x.data_ptr(), pv.data_ptr(), prec.data_ptr()
        out.noise_variance, out.effective_dof = noise.data_ptr(), dof.data_ptr()
        out.support_mask = mask.data_ptr() if mask is not None else None
        threshold = float(np.log(N / budget)) if budget is not None else 0.0
        out.support_threshold = threshold
        out.status = status.data_ptr()
        hist = np.zeros(max(1, self.cfg.max_iter) * len(nat.CG_HISTORY_COLUMNS), np.float32)
        info = nat.FbmeCgInfo()
        info.history = hist.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        with torch.cuda.device(self.device):
            rc = self.lib.fbme_cg_solve(self._plan, ctypes.c_void_p(y.data_ptr()),
                                        ctypes.c_void_p(probes.data_ptr()), ctypes.byref(out),
                                        ctypes.byref(info), ctypes.c_void_p(self._stream()))
        nat.check(rc, "fbme_cg_solve")
        it = int(info.iterations)
        cfg = self.cfg
        history: dict[str, list[float]] = {}
        if cfg.return_history:
            rows = hist[: it * 6].reshape(it, 6).astype(np.float64)
            for j, key in enumerate(nat.CG_HISTORY_COLUMNS):
                history[key] = rows[:, j].tolist()
            size, at = int(info.active_set_size), int(info.active_set_iteration)
            history["active_set_size"] = [float(size) if size and i + 1 >= at else 0.0 for i in range(it)]
            history["spatial_vertical_coupling"] = [float(cfg.spatial_coupling)] * it
            history["spatial_horizontal_coupling"] = [float(cfg.spatial_coupling)] * it
        report = cfg.return_history or cfg.eager_change_tracking or cfg.tol > 0.0 or cfg.verbose
        res = SBLResult(
            x=x, posterior_variance=pv, precision=prec, noise_variance=noise, effective_dof=dof,
            iterations=it, converged=bool(info.converged),
            relative_change=float(info.relative_change) if report else float("nan"),
            mode="dense" if self.dense else "cg", arithmetic_dtype="complex64", uamp_backend_used=None,
            active_set_size=int(info.active_set_size),
            support_mask=mask,
            support_score_threshold=(torch.full((B,), threshold, **f32) if budget is not None
                                     else None),
            history=history,
        )
        res.status = status
        return res

    # ------------------------------------------------------------- stages
    def matvec(self, prior: Tensor, noise: Tensor, v: Tensor) -> Tensor:
        """Q v for ``v`` complex64 ``[B, R, M]`` (R <= 1 + probes)."""
        B, R = v.shape[0], v.shape[1]
        v = v.contiguous()
        out = torch.empty_like(v)
        prior = prior.to(torch.float32).contiguous()
        noise = noise.to(torch.float32).contiguous()
        nat.check(self.lib.fbme_cg_matvec(self._plan, ctypes.c_void_p(prior.data_ptr()),
                                          ctypes.c_void_p(noise.data_ptr()),
                                          ctypes.c_void_p(v.data_ptr()), R,
                                          ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(self._stream())), "fbme_cg_matvec")
        return out

    def pcg(self, prior: Tensor, noise: Tensor, rhs: Tensor, tolerance: float,
            initial: Tensor | None = None) -> tuple[Tensor, int]:
        """Solve Q X = rhs (``[B, R, M]``); returns (X, loop iterations)."""
        R = rhs.shape[1]
        rhs = rhs.contiguous()
        sol = torch.empty_like(rhs)
        prior = prior.to(torch.float32).contiguous()
        noise = noise.to(torch.float32).contiguous()
        init = initial.contiguous() if initial is not None else None
        iters = ctypes.c_int32(0)
        nat.check(self.lib.fbme_pcg_solve(
            self._plan, ctypes.c_void_p(prior.data_ptr()), ctypes.c_void_p(noise.data_ptr()),
            ctypes.c_void_p(rhs.data_ptr()), R,
            ctypes.c_void_p(init.data_ptr()) if init is not None else None, float(tolerance),
            ctypes.c_void_p(sol.data_ptr()), ctypes.byref(iters),
            ctypes.c_void_p(self._stream())), "fbme_pcg_solve")
        return sol, int(iters.value)


def cg_sbl(tensor: Tensor, grid: Sequence[int], sample: Sequence[int], batch_shape: Sequence[int],
           cfg: SBLConfig, device: torch.device, dense: bool = False) -> SBLResult:
    """``fast_sbl`` with ``mode="cg"`` (or ``mode="dense"``) for ``tensor``
    ``[*batch, *sample]``."""
    batch = prod(batch_shape) if batch_shape else 1
    check_cg_supported(cfg, batch, dense)
    grid2 = tuple(grid) if len(grid) == 2 else (1, grid[0])
    sample2 = tuple(sample) if len(sample) == 2 else (1, sample[0])
    eng = CGEngine(batch, grid2, sample2, cfg, device, dense=dense)
    try:
        y = tensor.to(device=device, dtype=torch.complex64).reshape(batch, -1)
        res = eng.solve(y)
    finally:
        eng.close()
    shape = tuple(batch_shape) + tuple(grid)
    for name in ("x", "posterior_variance", "precision", "support_mask"):
        v = getattr(res, name)
        if v is not None:
            setattr(res, name, v.reshape(shape))
    for name in ("noise_variance", "effective_dof", "support_score_threshold"):
        v = getattr(res, name)
        if v is not None:
            setattr(res, name, v.reshape(tuple(batch_shape)))
    return res
