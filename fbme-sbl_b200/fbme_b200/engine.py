"""Host engine: one native FBME plan bound to torch-owned device buffers.

The engine resolves an ``SBLConfig`` into the C ABI's ``FbmeConfig``
(iteration budget, damping, active-set sizes), allocates the plan
workspace and every output as torch tensors on the target device, creates
the native plan, and launches replays on the current torch stream, so the
whole solve can be captured in a ``torch.cuda.CUDAGraph``.

Semantics follow the reference ``fast_sbl`` for ``mode="uamp"`` with the
active-set polish (torch_sbl/solver.py:925-2393): outputs are owned by the
engine and overwritten by the next run.
"""

from __future__ import annotations

import ctypes
from math import ceil, log, prod
from typing import Sequence

import torch
from torch import Tensor

from . import _native as nat
from .config import SBLConfig
from .result import SBLResult

BACKEND_NAME = "cuda-sm100a"


def uamp_iteration_limit(cfg: SBLConfig, n_grid: int, n_samples: int) -> int:
    """UAMP sweep budget (solver.py:1287-1309)."""
    minimum = max(cfg.min_iter, cfg.uamp_min_iter)
    limit = cfg.max_iter
    if cfg.uamp_auto_iterations:
        budget = ceil(cfg.uamp_iteration_offset + cfg.uamp_iteration_scale * n_grid / n_samples)
        limit = min(cfg.max_iter, max(minimum, budget))
    return limit


def fft_length_ok(n: int) -> bool:
    """Grid lengths the FP32 FFT stages take: 2^a or 3 * 2^a, 2 <= n <= 512."""
    n = int(n)
    if n < 2 or n > 512:
        return False
    if n % 3 == 0:
        n //= 3
    return n & (n - 1) == 0


def resolve_dft_terms(requested: int, grid: Sequence[int], uneven: bool = False) -> int:
    """The DFT stage form a plan runs: ``requested`` unless it is -1
    (automatic), which picks the FP32 FFT stages (0) for equal-shape plans
    whose grid lengths allow them and the 3-term tensor-core products
    otherwise (uneven plans: ``resolve_uneven_dft_terms``)."""
    if requested != -1:
        return int(requested)
    return 0 if not uneven and fft_length_ok(grid[0]) and fft_length_ok(grid[1]) else 3


def resolve_uneven_dft_terms(requested: int, grids: Sequence[Sequence[int]]) -> int:
    """The stage form of an uneven plan (one for all its buckets): the FP32
    FFT stages when every grid's lengths allow them, else the 3-term
    tensor-core products; an explicit ``requested`` wins."""
    if requested != -1:
        return int(requested)
    return 0 if all(fft_length_ok(g[0]) and fft_length_ok(g[1]) for g in grids) else 3


def resolve_native_config(cfg: SBLConfig, grid: Sequence[int], sample: Sequence[int],
                          n_observed: int | None = None, uneven: bool = False) -> nat.FbmeConfig:
    """Map the hot-path fields of ``cfg`` to ``FbmeConfig``.  Under an
    observation mask the sample count is the observed one
    (operator.n_samples in solver.py)."""
    n_grid = prod(grid)
    n_samples = prod(sample) if n_observed is None else int(n_observed)
    damping = cfg.uamp_damping
    if cfg.uamp_adaptive_damping:  # solver.py:1183-1189
        damping = max(damping, min(cfg.uamp_max_damping, 0.02 * n_grid / n_samples))
    k = min(cfg.uamp_polish_size, n_grid)
    exchange = min(cfg.uamp_polish_residual_exchange_size, max(k - 1, 0), n_grid - k)
    c = nat.FbmeConfig()
    c.uamp_iterations = uamp_iteration_limit(cfg, n_grid, n_samples)
    c.uamp_damping = damping
    c.damping = cfg.damping
    c.initialization_blend = cfg.initialization_blend if cfg.initialization == "backprojection" else -1.0
    c.initial_noise_fraction = cfg.initial_noise_fraction
    c.fixed_noise_variance = cfg.fixed_noise_variance if cfg.fixed_noise_variance is not None else 0.0
    c.min_variance = cfg.min_variance
    c.max_precision = cfg.max_precision
    c.hyper_shape = cfg.hyper_shape
    c.hyper_rate = cfg.hyper_rate
    c.noise_shape = cfg.noise_shape
    c.noise_rate = cfg.noise_rate
    c.noise_update = 1 if cfg.noise_update == "evidence" else 0
    c.polish_size = k
    c.polish_iterations = cfg.uamp_polish_iterations
    c.polish_prune_tail = int(cfg.uamp_polish_prune_tail)
    c.polish_reinitialize = int(cfg.uamp_polish_reinitialize)
    c.polish_evidence_gate = int(cfg.uamp_polish_evidence_gate)
    c.polish_damping = cfg.uamp_polish_damping
    c.evidence_margin_factor = cfg.uamp_polish_evidence_margin_factor
    c.exchange_size = exchange
    c.fixed_budget_diagnostics = int(cfg.uamp_polish_fixed_budget_diagnostics)
    c.cholesky_jitter_multiplier = cfg.cuda_cholesky_jitter_multiplier
    c.support_false_alarm_budget = (cfg.uamp_support_false_alarm_budget
                                    if cfg.uamp_support_false_alarm_budget is not None else 0.0)
    c.dft_terms = resolve_dft_terms(cfg.dft_terms, grid, uneven)
    return c


def check_supported(cfg: SBLConfig) -> None:
    """Reject configurations outside the built device path."""
    unsupported = {
        "joint_sparsity": cfg.joint_sparsity,
        "spatial_coupling": cfg.spatial_coupling > 0.0 or cfg.learn_spatial_coupling,
        "uamp_polish_support_prior": cfg.uamp_polish_support_prior,
        "uamp_polish_support_growth_steps": cfg.uamp_polish_support_growth_steps != 0,
        "uamp_polish_support_shrink_steps": cfg.uamp_polish_support_shrink_steps != 0,
        "uamp_polish_coordinate_steps": cfg.uamp_polish_coordinate_steps != 0,
        "uamp_polish_noise_coordinate_steps": cfg.uamp_polish_noise_coordinate_steps != 0,
        "uamp_polish_high_precision": cfg.uamp_polish_high_precision,
        "uamp_polish_max_truncation_delta": cfg.uamp_polish_max_truncation_delta is not None,
        "offgrid_refinement": cfg.offgrid_refinement,
    }
    bad = [k for k, v in unsupported.items() if v]
    if bad:
        raise NotImplementedError("the B200 FBME path does not implement: " + ", ".join(bad))
    if cfg.tol > 0.0:
        raise NotImplementedError(
            "mode='uamp' runs the fixed UAMP budget on the device; set tol=0 "
            "(every UAMP preset does)")
    if cfg.uamp_polish_global_certificate and (
            cfg.uamp_polish_iterations + cfg.uamp_polish_support_repairs > 8):
        raise NotImplementedError(
            "the device certificate keeps at most 8 evidence values: "
            "uamp_polish_iterations + uamp_polish_support_repairs <= 8")
    if cfg.uamp_polish_size < 1 or not cfg.uamp_polish_prune_tail:
        raise NotImplementedError(
            "the device UAMP path implements the zero-tail active-set polish "
            "(uamp_polish_size >= 1 and uamp_polish_prune_tail=True, as in the FBME presets)")


def ratio_threshold_for_evidence_tolerance(tolerance: float) -> float:
    """The rho >= 1 with rho - 1 - log(rho) = tolerance, the inactive-ratio
    form of the stationarity tolerance (torch_sbl/solver.py:3499-3519): an
    upper bound by doubling, then 64 bisection steps."""
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


class FBMEEngine:
    """A native plan for ``batch`` scenes of one shape and configuration."""

    def __init__(self, batch: int, grid: Sequence[int], sample: Sequence[int], cfg: SBLConfig,
                 device: torch.device, stream: torch.cuda.Stream | None = None,
                 n_tile: int | None = None, observation_mask: Tensor | None = None) -> None:
        self.lib = nat.lib()
        if device.type != "cuda":
            raise RuntimeError("the FBME B200 engine needs a CUDA device")
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.batch = int(batch)
        self.grid = tuple(int(v) for v in grid)
        self.sample = tuple(int(v) for v in sample)
        self.cfg = cfg
        self.n_grid, self.n_samples = prod(self.grid), prod(self.sample)
        # observation mask (operators.py:57-75): [M1, M2] bool, shared by the batch
        self.mask = None
        n_observed = None
        if observation_mask is not None:
            m = torch.as_tensor(observation_mask, device=device, dtype=torch.bool)
            if tuple(m.shape) != self.sample:
                raise ValueError(f"observation_mask must have shape {self.sample}, got {tuple(m.shape)}.")
            n_observed = int(m.sum())
            if n_observed == 0:
                raise ValueError("observation_mask must retain at least one sample.")
            self.mask = m.to(torch.uint8).contiguous()
        self.n_observed = self.n_samples if n_observed is None else n_observed
        self.native_cfg = resolve_native_config(cfg, self.grid, self.sample, n_observed)
        shapes = (nat.FbmeShape * self.batch)()
        for i in range(self.batch):
            shapes[i] = nat.FbmeShape(self.grid[0], self.grid[1], self.sample[0], self.sample[1])
        self._shapes = shapes
        # the DFT stage tile width (None: chosen from the batch's tile count)
        if n_tile is None:
            from .autotune import default_width

            n_tile = default_width(self.grid, self.sample, self.batch, int(self.native_cfg.dft_terms),
                                   torch.cuda.get_device_properties(device).multi_processor_count)
        self.n_tile = n_tile
        self._params = nat.FbmeShapeParams(shapes[0], 0, -1.0, -1, int(n_tile or 0))
        nbytes = self.lib.fbme_plan_workspace_bytes_ex(shapes, self.batch, ctypes.byref(self.native_cfg),
                                                       ctypes.byref(self._params), 1)
        if nbytes == 0:
            nat.check(nat.FBME_ERR_INVALID, "fbme_plan_workspace_bytes")
        self.workspace = torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=device)
        base = self.workspace.data_ptr()
        self._ws_ptr = (base + 255) & ~255
        B, N, K = self.batch, self.n_grid, self.native_cfg.polish_size
        P = self.native_cfg.polish_iterations
        self.certify = bool(cfg.uamp_polish_global_certificate)
        R = int(cfg.uamp_polish_support_repairs) if self.certify else 0
        f32 = dict(dtype=torch.float32, device=device)
        self.out = {
            "x": torch.zeros(B, N, dtype=torch.complex64, device=device),
            "posterior_variance": torch.zeros(B, N, **f32),
            "precision": torch.zeros(B, N, **f32),
            "support_mask": torch.zeros(B, N, dtype=torch.bool, device=device),
            "noise_variance": torch.zeros(B, **f32),
            "effective_dof": torch.zeros(B, **f32),
            "negative_log_evidence": torch.zeros(B, **f32),
            "evidence_trace": torch.zeros(B, P + R, **f32),
            "support_exchanges_accepted": torch.zeros(B, dtype=torch.int64, device=device),
            "fixed_budget_gamma_residual": torch.zeros(B, **f32),
            "fixed_budget_noise_residual": torch.zeros(B, **f32),
            "fixed_budget_objective_decrease": torch.zeros(B, **f32),
            "fixed_budget_monotone": torch.zeros(B, dtype=torch.bool, device=device),
            "support_score_threshold": torch.zeros(B, **f32),
            "active_indices": torch.zeros(B, K, dtype=torch.int64, device=device),
            "active_values": torch.zeros(B, K, dtype=torch.complex64, device=device),
            "status": torch.zeros(B, dtype=torch.int32, device=device),
        }
        o = nat.FbmeOutputs()
        for name, _ in nat.FbmeOutputs._fields_:
            setattr(o, name, self.out[name].data_ptr())
        self._outputs = o
        self._plan = ctypes.c_void_p()
        st = stream or torch.cuda.current_stream(device)
        with torch.cuda.device(device):
            rc = self.lib.fbme_plan_create_ex(shapes, self.batch, ctypes.byref(self.native_cfg),
                                              ctypes.byref(self._params), 1, ctypes.c_void_p(self._ws_ptr),
                                              ctypes.c_size_t(nbytes), ctypes.c_void_p(st.cuda_stream),
                                              ctypes.byref(self._plan))
        nat.check(rc, "fbme_plan_create")
        if self.mask is not None:
            with torch.cuda.device(device):
                rc = self.lib.fbme_plan_set_observation_mask(self._plan, ctypes.c_void_p(self.mask.data_ptr()),
                                                             ctypes.c_void_p(st.cuda_stream))
            nat.check(rc, "fbme_plan_set_observation_mask")
        if self.certify:
            self._set_certificate(R)
        # constant result fields of the zero-tail polish (solver.py:4052-4068, 4639-4653)
        self._false = torch.zeros(B, dtype=torch.bool, device=device)
        self._true = torch.ones(B, dtype=torch.bool, device=device)
        self._zero = torch.zeros(B, **f32)

    def _set_certificate(self, repairs: int) -> None:
        """Device outputs of the global certificate and support repairs
        (solver.py:4511-4628, 4851-4870, 5388-5460), registered with the plan."""
        cfg, B, dev = self.cfg, self.batch, self.device
        fwer = cfg.uamp_polish_familywise_error_rate
        inactive = max(self.n_grid - int(self.native_cfg.polish_size), 1)
        self.fw_threshold = log(inactive / fwer) if fwer is not None else None
        self.stationarity_threshold = ratio_threshold_for_evidence_tolerance(
            cfg.uamp_polish_coordinate_tolerance)
        floats = ("inactive_max_evidence_ratio", "inactive_evidence_gain", "inactive_optimal_variance",
                  "active_max_evidence_gain", "active_optimal_variance", "active_max_deletion_gain",
                  "active_penalized_evidence_gain")
        ints = ("inactive_best_index", "support_repairs_accepted", "active_best_index")
        flags = ("coordinate_stationary", "type2_map_coordinate_stationary", "familywise_no_discovery")
        self.cert = {k: torch.zeros(B, dtype=torch.float32, device=dev) for k in floats}
        self.cert.update({k: torch.zeros(B, dtype=torch.int64, device=dev) for k in ints})
        self.cert.update({k: torch.zeros(B, dtype=torch.bool, device=dev) for k in flags})
        c = nat.FbmeCertificate()
        c.support_repairs = repairs
        c.coordinate_tolerance = cfg.uamp_polish_coordinate_tolerance
        c.familywise_ratio_threshold = self.fw_threshold if self.fw_threshold is not None else 0.0
        for name, _ in nat.FbmeCertificate._fields_[3:-2]:
            setattr(c, name, self.cert[name].data_ptr())
        nbytes = int(self.lib.fbme_plan_certificate_workspace_bytes(self._plan))
        self._cert_ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        c.workspace = (self._cert_ws.data_ptr() + 255) & ~255
        c.workspace_bytes = nbytes
        self._certificate = c
        nat.check(self.lib.fbme_plan_set_certificate(self._plan, ctypes.byref(c)), "fbme_plan_set_certificate")

    # ------------------------------------------------------------------ runs
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def run(self, y: Tensor) -> None:
        """Solve ``y`` ([B, M1*M2] or any contiguous complex64 view of it)."""
        self._check_y(y)
        nat.check(self.lib.fbme_plan_replay(self._plan, ctypes.c_void_p(y.data_ptr()),
                                            ctypes.byref(self._outputs),
                                            ctypes.c_void_p(self._stream())), "fbme_plan_replay")

    def run_uamp(self, y: Tensor) -> None:
        self._check_y(y)
        nat.check(self.lib.fbme_uamp_run(self._plan, ctypes.c_void_p(y.data_ptr()),
                                         ctypes.c_void_p(self._stream())), "fbme_uamp_run")

    def run_polish(self, y: Tensor) -> None:
        self._check_y(y)
        nat.check(self.lib.fbme_polish_run(self._plan, ctypes.c_void_p(y.data_ptr()),
                                           ctypes.byref(self._outputs),
                                           ctypes.c_void_p(self._stream())), "fbme_polish_run")

    def profile(self, y: Tensor) -> dict[str, tuple[float, int]]:
        """One eagerly launched replay with CUDA events around every kernel:
        {group name: (device ms summed over launches, launches)}."""
        self._check_y(y)
        n = nat.NUM_GROUPS
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int32 * n)()
        nat.check(self.lib.fbme_plan_profile(self._plan, ctypes.c_void_p(y.data_ptr()),
                                             ctypes.byref(self._outputs),
                                             ctypes.c_void_p(self._stream()), ms, cnt, n),
                  "fbme_plan_profile")
        return {self.lib.fbme_profile_group_name(g).decode(): (float(ms[g]), int(cnt[g]))
                for g in range(n)}

    def dft_forward(self, coeff: Tensor) -> Tensor:
        """A(X) for [B, N] complex64 coefficients -> [B, M] data."""
        self._check(coeff, self.n_grid)
        out = torch.empty(self.batch, self.n_samples, dtype=torch.complex64, device=self.device)
        nat.check(self.lib.fbme_dft_forward(self._plan, ctypes.c_void_p(coeff.data_ptr()),
                                            ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(self._stream())), "fbme_dft_forward")
        return out

    def dft_adjoint(self, data: Tensor) -> Tensor:
        """A^H(Y) for [B, M] complex64 data -> [B, N] coefficients."""
        self._check(data, self.n_samples)
        out = torch.empty(self.batch, self.n_grid, dtype=torch.complex64, device=self.device)
        nat.check(self.lib.fbme_dft_adjoint(self._plan, ctypes.c_void_p(data.data_ptr()),
                                            ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(self._stream())), "fbme_dft_adjoint")
        return out

    def state(self) -> dict[str, Tensor]:
        """Views of the resident UAMP state (for tests and tools)."""
        st = nat.FbmeState()
        nat.check(self.lib.fbme_plan_state(self._plan, ctypes.byref(st)), "fbme_plan_state")
        B, N, M = self.batch, self.n_grid, self.n_samples

        def view(ptr: int, shape, dtype):
            ws0 = self.workspace.data_ptr()
            itemsize = torch.empty((), dtype=dtype).element_size()
            off = ptr - ws0
            n = prod(shape)
            flat = self.workspace[off: off + n * itemsize].view(dtype)
            return flat.view(*shape)

        return {
            "mean": view(st.mean, (B, N), torch.complex64),
            "variance": view(st.variance, (B, N), torch.float32),
            "prior_variance": view(st.prior_variance, (B, N), torch.float32),
            "backprojection": view(st.backprojection, (B, N), torch.complex64),
            "prediction": view(st.prediction, (B, M), torch.complex64),
            "noise_variance": view(st.noise_variance, (B,), torch.float32),
            "data_variance": view(st.data_variance, (B,), torch.float32),
        }

    def _check(self, t: Tensor, length: int) -> None:
        if (t.device != self.device or t.dtype != torch.complex64 or not t.is_contiguous()
                or t.numel() != self.batch * length):
            raise ValueError(f"expected a contiguous complex64 tensor of {self.batch}x{length} "
                             f"elements on {self.device}")

    def _check_y(self, y: Tensor) -> None:
        self._check(y, self.n_samples)

    # --------------------------------------------------------------- results
    def result(self, batch_shape: tuple[int, ...]) -> SBLResult:
        """Engine-owned ``SBLResult`` views shaped like the reference's."""
        o, cfg = self.out, self.cfg
        out_shape = (*batch_shape, *self.grid)
        K = self.native_cfg.polish_size
        exch = o["support_exchanges_accepted"].reshape(batch_shape) \
            if self.native_cfg.exchange_size > 0 else None
        fb = bool(self.native_cfg.fixed_budget_diagnostics)
        has_mask = cfg.uamp_support_false_alarm_budget is not None
        nle = o["negative_log_evidence"].reshape(batch_shape)
        extra = self._certificate_fields(batch_shape) if self.certify else {}
        if self.certify:  # residual exchanges and repairs share one counter
            exch = extra.pop("support_repairs_accepted")
        return SBLResult(
            **extra,
            x=o["x"].reshape(out_shape),
            posterior_variance=o["posterior_variance"].reshape(out_shape),
            precision=o["precision"].reshape(out_shape),
            noise_variance=o["noise_variance"].reshape(batch_shape),
            effective_dof=o["effective_dof"].reshape(batch_shape),
            iterations=int(self.native_cfg.uamp_iterations),
            converged=False,
            relative_change=float("nan"),
            mode="uamp",
            arithmetic_dtype="complex64",
            uamp_backend_used=BACKEND_NAME,
            active_set_size=K,
            negative_log_evidence=nle,
            evidence_trace=o["evidence_trace"],
            hard_pruning_accepted=self._false.reshape(batch_shape),
            truncation_certified=self._false.reshape(batch_shape),
            support_repairs_accepted=exch,
            support_exchanges_accepted=exch,
            active_model_selected=self._true.reshape(batch_shape),
            support_log_odds_penalty=self._zero.reshape(batch_shape),
            penalized_negative_log_evidence=nle,
            penalized_evidence_trace=o["evidence_trace"],
            fixed_budget_gamma_residual=o["fixed_budget_gamma_residual"].reshape(batch_shape) if fb else None,
            fixed_budget_noise_residual=o["fixed_budget_noise_residual"].reshape(batch_shape) if fb else None,
            fixed_budget_objective_decrease=(
                o["fixed_budget_objective_decrease"].reshape(batch_shape) if fb else None),
            fixed_budget_monotone=o["fixed_budget_monotone"].reshape(batch_shape) if fb else None,
            support_mask=o["support_mask"].reshape(out_shape) if has_mask else None,
            support_score_threshold=(o["support_score_threshold"].reshape(batch_shape)
                                     if has_mask else None),
            status=o["status"].reshape(batch_shape),
        )

    def _certificate_fields(self, batch_shape: tuple[int, ...]) -> dict:
        """The certificate's result fields (solver.py:2196-2330), with the
        support log-odds penalty zero (no support prior)."""
        c = {k: v.reshape(batch_shape) for k, v in self.cert.items()}
        thr = torch.full(batch_shape, self.stationarity_threshold, dtype=torch.float32, device=self.device)
        f = dict(
            inactive_max_evidence_ratio=c["inactive_max_evidence_ratio"],
            inactive_best_index=c["inactive_best_index"],
            inactive_evidence_gain=c["inactive_evidence_gain"],
            inactive_optimal_variance=c["inactive_optimal_variance"],
            support_repairs_accepted=c["support_repairs_accepted"],
            active_max_evidence_gain=c["active_max_evidence_gain"],
            active_best_index=c["active_best_index"],
            active_optimal_variance=c["active_optimal_variance"],
            active_max_deletion_gain=c["active_max_deletion_gain"],
            coordinate_stationary=c["coordinate_stationary"],
            type2_coordinate_stationary=c["coordinate_stationary"],
            inactive_ratio_threshold=thr,
            stationarity_ratio_threshold=thr,
            inactive_penalized_evidence_gain=c["inactive_evidence_gain"],
            active_penalized_evidence_gain=c["active_penalized_evidence_gain"],
            type2_map_coordinate_stationary=c["type2_map_coordinate_stationary"],
        )
        if self.fw_threshold is not None:
            f.update(familywise_ratio_threshold=torch.full(batch_shape, self.fw_threshold, dtype=torch.float32,
                                                           device=self.device),
                     familywise_no_discovery=c["familywise_no_discovery"],
                     familywise_support_certified=c["familywise_no_discovery"])
        return f

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None and self._plan.value:
            self.lib.fbme_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------ stand-alone kernels
def _tensor_contract(name: str, tensor: Tensor, *, dtype: torch.dtype, shape: tuple[int, ...],
                     device: torch.device | None = None) -> None:
    """The raw-pointer contract of the stand-alone kernels, with the
    reference's messages (torch_sbl/triton_kernels.py:451-473)."""
    if not tensor.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor.")
    if tensor.dtype != dtype:
        raise ValueError(f"{name} must have dtype {dtype}.")
    if tuple(tensor.shape) != shape:
        raise ValueError(f"{name} must have shape {shape}, got {tuple(tensor.shape)}.")
    if not tensor.is_contiguous():
        raise ValueError(f"{name} must be C-contiguous.")
    if device is not None and tensor.device != device:
        raise ValueError(f"{name} must be on {device}, got {tensor.device}.")


def uamp_prior_update(mean: Tensor, posterior_variance: Tensor, old_prior: Tensor, prior_floor: Tensor, *,
                      hyper_shape: float, hyper_rate: float, damping: float, maximum: float) -> Tensor:
    """The unfused variational ARD update of one UAMP iteration, as
    torch_sbl/triton_kernels.py:670-735 (uamp_prior_update): same arguments,
    contract and errors; runs the library's fbme_uamp_prior_update kernel."""
    if old_prior.ndim != 2:
        raise ValueError("old_prior must have shape [B, N].")
    batch_size, n_grid = old_prior.shape
    dev = old_prior.device
    _tensor_contract("mean", mean, dtype=torch.complex64, shape=(batch_size, n_grid), device=dev)
    for name, t in (("posterior_variance", posterior_variance), ("old_prior", old_prior)):
        _tensor_contract(name, t, dtype=torch.float32, shape=(batch_size, n_grid), device=dev)
    _tensor_contract("prior_floor", prior_floor, dtype=torch.float32, shape=(batch_size,), device=dev)
    out = torch.empty_like(old_prior)
    lib = nat.lib()
    with torch.cuda.device(dev):
        rc = lib.fbme_uamp_prior_update(
            ctypes.c_void_p(mean.data_ptr()), ctypes.c_void_p(posterior_variance.data_ptr()),
            ctypes.c_void_p(old_prior.data_ptr()), ctypes.c_void_p(prior_floor.data_ptr()), batch_size, n_grid,
            float(hyper_shape), float(hyper_rate), float(damping), float(maximum),
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    nat.check(rc, "fbme_uamp_prior_update")
    return out
