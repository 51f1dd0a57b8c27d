"""Uneven batches: scenes of different shapes in one native plan.

The reference batches only equal shapes, through leading dimensions
(torch_sbl/solver.py:966-1001); a caller with scenes of several shapes
builds one plan per shape and replays them one after another.
``UnevenEngine`` binds one native plan over a list of scene shapes.  The
library groups the scenes into one bucket per shape (in order of first
appearance), each with the state and tables of an equal-shape batch.  The
shape-dependent values -- the UAMP sweep budget T_u (solver.py:1295-1309),
the adaptive damping (solver.py:1183-1189), the resolved exchange size and
the tuned DFT tile width -- are set per bucket, so a scene stops after its
own shape's T_u sweeps.  Each UAMP step is one launch over all buckets (up
to 64 per launch); each bucket's polish runs on its own stream; a gather and
a scatter kernel map the packed scene-order buffers to bucket order and
back.  Every scene's result equals that of an equal-shape plan bit for bit.

Inputs and outputs are packed: scene i's M1*M2 samples (N1*N2 pixels)
follow scene i-1's.  ``UnevenSBLPlan`` captures the whole uneven solve in
one CUDA graph, with the same replay semantics as the fixed-shape plans:
graph-owned results, overwritten by the next replay.
"""

from __future__ import annotations

import ctypes
import dataclasses
from math import prod
from typing import Sequence

import torch
from torch import Tensor

from . import _native as nat
from .config import SBLConfig, fbme_profile_config
from .engine import BACKEND_NAME, check_supported, resolve_native_config, resolve_uneven_dft_terms
from .result import SBLResult

Shape = tuple[tuple[int, int], tuple[int, int]]


def _shape(grid: Sequence[int], sample: Sequence[int]) -> Shape:
    g = tuple(int(v) for v in grid)
    s = tuple(int(v) for v in sample)
    if len(g) != 2 or len(s) != 2:
        raise ValueError("uneven plans take 2-D grids (N1, N2) and samples (M1, M2)")
    if any(m < 1 or m > n for m, n in zip(s, g)):
        raise ValueError("Each sample dimension must satisfy 0 < M <= N.")
    return g, s


class UnevenEngine:
    """One native plan over scenes of (possibly) different shapes."""

    def __init__(self, shapes: Sequence[tuple[Sequence[int], Sequence[int]]], cfg: SBLConfig,
                 device: torch.device, *, tile_widths: dict[Shape, int] | None = None,
                 stream: torch.cuda.Stream | None = None) -> None:
        if device.type != "cuda":
            raise RuntimeError("the FBME B200 engine needs a CUDA device")
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        if not shapes:
            raise ValueError("an uneven plan needs at least one scene")
        check_supported(cfg)
        self.lib = nat.lib()
        self.device = device
        self.cfg = cfg
        self.scenes: list[Shape] = [_shape(g, s) for g, s in shapes]
        self.batch = len(self.scenes)
        tile_widths = tile_widths or {}
        pix = [prod(g) for g, _ in self.scenes]
        smp = [prod(s) for _, s in self.scenes]
        self.pix_off = [0]
        self.smp_off = [0]
        for p, m in zip(pix, smp):
            self.pix_off.append(self.pix_off[-1] + p)
            self.smp_off.append(self.smp_off[-1] + m)
        self.total_pixels, self.total_samples = self.pix_off[-1], self.smp_off[-1]

        # the shape-dependent values, resolved per distinct shape
        distinct: list[Shape] = []
        for sh in self.scenes:
            if sh not in distinct:
                distinct.append(sh)
        terms = resolve_uneven_dft_terms(int(cfg.dft_terms), [sh[0] for sh in distinct])
        cfg_t = dataclasses.replace(cfg, dft_terms=terms)
        resolved = {sh: resolve_native_config(cfg_t, sh[0], sh[1], uneven=True) for sh in distinct}
        base = resolved[self.scenes[0]]
        if len({(r.polish_size, r.polish_iterations) for r in resolved.values()}) != 1:
            raise ValueError("every scene of an uneven plan needs N1*N2 >= polish_size")
        self.native_cfg = base
        self.shape_iterations = {sh: int(r.uamp_iterations) for sh, r in resolved.items()}
        shape_arr = (nat.FbmeShape * self.batch)()
        for i, (g, s) in enumerate(self.scenes):
            shape_arr[i] = nat.FbmeShape(g[0], g[1], s[0], s[1])
        params = (nat.FbmeShapeParams * len(distinct))()
        # the buckets run concurrently, so the narrow-tile default applies
        # only when all of them together leave SMs idle
        from .autotune import candidates, default_width, stage_tiles

        sms = torch.cuda.get_device_properties(device).multi_processor_count
        fill = sum(sum(stage_tiles(sh[0], sh[1], max(candidates(sh[0], sh[1], terms) or [256])))
                   for sh in self.scenes)
        self.tile_widths = {sh: int(tile_widths.get(sh) or default_width(sh[0], sh[1], 1, terms,
                                                                         sms if fill < sms else 0))
                            for sh in distinct}
        for i, sh in enumerate(distinct):
            r = resolved[sh]
            params[i] = nat.FbmeShapeParams(nat.FbmeShape(sh[0][0], sh[0][1], sh[1][0], sh[1][1]),
                                            r.uamp_iterations, r.uamp_damping, r.exchange_size,
                                            self.tile_widths[sh])
        self._shape_arr, self._params = shape_arr, params
        nbytes = self.lib.fbme_plan_workspace_bytes_ex(shape_arr, self.batch, ctypes.byref(base), params,
                                                       len(distinct))
        if nbytes == 0:
            nat.check(nat.FBME_ERR_INVALID, "fbme_plan_workspace_bytes_ex")
        self.workspace = torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=device)
        ws = (self.workspace.data_ptr() + 255) & ~255

        B, K, P = self.batch, base.polish_size, base.polish_iterations
        NP = self.total_pixels
        f32 = dict(dtype=torch.float32, device=device)
        self.out = {
            "x": torch.zeros(NP, dtype=torch.complex64, device=device),
            "posterior_variance": torch.zeros(NP, **f32),
            "precision": torch.zeros(NP, **f32),
            "support_mask": torch.zeros(NP, dtype=torch.bool, device=device),
            "noise_variance": torch.zeros(B, **f32),
            "effective_dof": torch.zeros(B, **f32),
            "negative_log_evidence": torch.zeros(B, **f32),
            "evidence_trace": torch.zeros(B, P, **f32),
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
            rc = self.lib.fbme_plan_create_ex(shape_arr, self.batch, ctypes.byref(base), params,
                                              len(distinct), ctypes.c_void_p(ws), ctypes.c_size_t(nbytes),
                                              ctypes.c_void_p(st.cuda_stream), ctypes.byref(self._plan))
        nat.check(rc, "fbme_plan_create_ex")
        self._false = torch.zeros(B, dtype=torch.bool, device=device)
        self._true = torch.ones(B, dtype=torch.bool, device=device)
        self._zero = torch.zeros(B, **f32)

    # ------------------------------------------------------------------ runs
    def run(self, y: Tensor) -> None:
        """Solve the packed samples ``y`` (complex64, sum of M1*M2 values)."""
        if (y.device != self.device or y.dtype != torch.complex64 or not y.is_contiguous()
                or y.numel() != self.total_samples):
            raise ValueError(f"expected a contiguous complex64 tensor of {self.total_samples} packed "
                             f"samples on {self.device}")
        st = torch.cuda.current_stream(self.device).cuda_stream
        nat.check(self.lib.fbme_plan_replay(self._plan, ctypes.c_void_p(y.data_ptr()),
                                            ctypes.byref(self._outputs), ctypes.c_void_p(st)),
                  "fbme_plan_replay")

    def profile(self, y: Tensor) -> dict[str, tuple[float, int]]:
        """One eager solve, buckets in sequence, with CUDA events around
        every launch: {group name: (device ms, launches)}."""
        n = nat.NUM_GROUPS
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int32 * n)()
        st = torch.cuda.current_stream(self.device).cuda_stream
        nat.check(self.lib.fbme_plan_profile(self._plan, ctypes.c_void_p(y.data_ptr()),
                                             ctypes.byref(self._outputs), ctypes.c_void_p(st), ms, cnt, n),
                  "fbme_plan_profile")
        return {self.lib.fbme_profile_group_name(g).decode(): (float(ms[g]), int(cnt[g])) for g in range(n)}

    def buckets(self) -> list[dict]:
        """The plan's buckets: shape, scene count and resolved values."""
        out = []
        for b in range(self.lib.fbme_plan_bucket_count(self._plan)):
            q = nat.FbmeShapeParams()
            n = ctypes.c_int32()
            nat.check(self.lib.fbme_plan_bucket(self._plan, b, ctypes.byref(q), ctypes.byref(n)),
                      "fbme_plan_bucket")
            out.append(dict(grid=(q.shape.n1, q.shape.n2), sample=(q.shape.m1, q.shape.m2), scenes=n.value,
                            uamp_iterations=q.uamp_iterations, uamp_damping=q.uamp_damping,
                            exchange_size=q.exchange_size, dft_n_tile=q.dft_n_tile))
        return out

    def pack(self, data: Sequence[Tensor], out: Tensor | None = None) -> Tensor:
        """Scene tensors ([M1, M2] each) packed into one contiguous buffer."""
        if len(data) != self.batch:
            raise ValueError(f"expected {self.batch} scenes, got {len(data)}")
        for i, (d, (_, s)) in enumerate(zip(data, self.scenes)):
            if tuple(d.shape) != s:
                raise ValueError(f"scene {i}: expected samples of shape {s}, got {tuple(d.shape)}")
        flat = [d.reshape(-1) for d in data]
        if out is None:
            return torch.cat(flat)
        torch.cat(flat, out=out)
        return out

    # --------------------------------------------------------------- results
    def results(self) -> list[SBLResult]:
        """Engine-owned per-scene ``SBLResult`` views (0-d scalars)."""
        o, cfg, nc = self.out, self.cfg, self.native_cfg
        fb = bool(nc.fixed_budget_diagnostics)
        has_mask = cfg.uamp_support_false_alarm_budget is not None
        res = []
        for i, (g, s) in enumerate(self.scenes):
            p0, p1 = self.pix_off[i], self.pix_off[i + 1]
            exch = o["support_exchanges_accepted"][i] if nc.exchange_size > 0 else None
            nle = o["negative_log_evidence"][i]
            res.append(SBLResult(
                x=o["x"][p0:p1].view(g),
                posterior_variance=o["posterior_variance"][p0:p1].view(g),
                precision=o["precision"][p0:p1].view(g),
                noise_variance=o["noise_variance"][i],
                effective_dof=o["effective_dof"][i],
                iterations=self.shape_iterations[(g, s)],
                converged=False,
                relative_change=float("nan"),
                mode="uamp",
                arithmetic_dtype="complex64",
                uamp_backend_used=BACKEND_NAME,
                active_set_size=int(nc.polish_size),
                negative_log_evidence=nle,
                evidence_trace=o["evidence_trace"][i],
                hard_pruning_accepted=self._false[i],
                truncation_certified=self._false[i],
                support_repairs_accepted=exch,
                support_exchanges_accepted=exch,
                active_model_selected=self._true[i],
                support_log_odds_penalty=self._zero[i],
                penalized_negative_log_evidence=nle,
                penalized_evidence_trace=o["evidence_trace"][i],
                fixed_budget_gamma_residual=o["fixed_budget_gamma_residual"][i] if fb else None,
                fixed_budget_noise_residual=o["fixed_budget_noise_residual"][i] if fb else None,
                fixed_budget_objective_decrease=o["fixed_budget_objective_decrease"][i] if fb else None,
                fixed_budget_monotone=o["fixed_budget_monotone"][i] if fb else None,
                support_mask=o["support_mask"][p0:p1].view(g) if has_mask else None,
                support_score_threshold=o["support_score_threshold"][i] if has_mask else None,
                status=o["status"][i],
            ))
        return res

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None and self._plan.value:
            self.lib.fbme_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


class UnevenSBLPlan:
    """A captured FBME solve of scenes with different shapes.

    ``examples`` are the scenes' CUDA complex64 samples ([M1, M2] each) and
    ``grid_shapes`` their (N1, N2) grids.  ``profile`` picks the FBME-Stable
    or FBME-Fast configuration.  With ``tune=True`` the DFT tile width of
    every shape comes from the autotuner (measured once, then cached).
    """

    def __init__(self, examples: Sequence[Tensor], grid_shapes: Sequence[Sequence[int]], *,
                 profile: str = "stable", polish_size: int = 32, warmup: int = 3, tune: bool = False,
                 config: SBLConfig | None = None, tile_widths: dict[Shape, int] | None = None) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA Graph execution requires CUDA.")
        if len(examples) != len(grid_shapes) or not examples:
            raise ValueError("one grid shape per example scene is required")
        if warmup < 1:
            raise ValueError("warmup must be positive.")
        dev = examples[0].device
        for d in examples:
            if not isinstance(d, Tensor) or not d.is_cuda or d.device != dev:
                raise ValueError("examples must be CUDA tensors on one device.")
            if d.dtype != torch.complex64:
                raise ValueError("the B200 FBME plans compute in complex64; pass complex64 data.")
            if d.ndim != 2:
                raise ValueError("each example is one scene's [M1, M2] samples")
        self.device = dev
        self.profile = profile
        self.config = config if config is not None else fbme_profile_config(profile, polish_size)
        self.config.validate()
        shapes = [(tuple(g), tuple(d.shape)) for g, d in zip(grid_shapes, examples)]
        if tune:
            from .autotune import tune_shapes

            tile_widths = {**tune_shapes(shapes, self.config, dev), **(tile_widths or {})}
        self._engine = UnevenEngine(shapes, self.config, dev, tile_widths=tile_widths)
        self.input_buffer = torch.empty(self._engine.total_samples, dtype=torch.complex64, device=dev)
        self._engine.pack(examples, out=self.input_buffer)

        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self._engine.run(self.input_buffer)
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self._graph = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(self._graph):
                self._engine.run(self.input_buffer)
        except Exception as error:
            raise RuntimeError("CUDA Graph capture failed for this uneven plan.") from error
        self._results = self._engine.results()

    @property
    def result(self) -> list[SBLResult]:
        return self._results

    @property
    def engine(self) -> UnevenEngine:
        return self._engine

    def buckets(self) -> list[dict]:
        return self._engine.buckets()

    def replay(self, data: Sequence[Tensor] | Tensor | None = None, *,
               synchronize: bool = False) -> list[SBLResult]:
        """Replay the captured solve.  ``data``: a list of per-scene [M1, M2]
        tensors, or one packed complex64 tensor of all samples."""
        if data is not None:
            if isinstance(data, Tensor):
                if data.device != self.device or data.dtype != torch.complex64 or \
                        data.numel() != self._engine.total_samples:
                    raise ValueError("packed replay data must be complex64 with every scene's samples "
                                     f"({self._engine.total_samples}) on {self.device}")
                self.input_buffer.copy_(data.reshape(-1))
            else:
                for d in data:
                    if not isinstance(d, Tensor) or d.device != self.device or d.dtype != torch.complex64:
                        raise ValueError(f"replay data must be complex64 CUDA tensors on {self.device}")
                self._engine.pack(data, out=self.input_buffer)
        self._graph.replay()
        if synchronize:
            torch.cuda.synchronize(self.device)
        return self._results


def make_uneven_plan(examples: Sequence[Tensor], grid_shapes: Sequence[Sequence[int]], *,
                     profile: str = "stable", polish_size: int = 32, warmup: int = 3,
                     tune: bool = False) -> UnevenSBLPlan:
    """Build a captured FBME plan over scenes of different shapes."""
    return UnevenSBLPlan(examples, grid_shapes, profile=profile, polish_size=polish_size, warmup=warmup,
                         tune=tune)
