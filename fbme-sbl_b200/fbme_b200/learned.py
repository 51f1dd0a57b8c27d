"""Learned warm start of the FBME plans (no counterpart in the reference).

A 3-layer 3x3 convolutional network (8 hidden channels, 809 parameters;
BF16 operands, FP32 accumulation; csrc/cnn.cu) maps the
features of the backprojection A^H y to the log of the initial prior
variance relative to the uniform level P/N (P the data power).  It replaces
the backprojection-blend initialisation of torch_sbl/solver.py:1072-1099;
with it the plan runs fewer UAMP sweeps.

Training pairs come from the plain solver itself: the network's default
target is the plain plan's final answer, log(|x|^2 / (P/N) + 1e-3) of its
polished reconstruction x, clamped to [-20, 20]; so the network learns
where plain FBME puts its atoms, and the warm-started plan reaches the
same atoms with fewer sweeps.  Training
runs on the GPU with the library's own forward, backward and Adam kernels.

``LearnedSBLPlan`` replays the warm-started plan and keeps plain FBME as the
fallback: a scene whose warm-started solve fails the evidence / residual
check (finite, monotone evidence trace; fixed-point residuals of the prior
and noise below the plain solver's calibrated bounds) is solved again by
the plain plan, whose result is returned for it.
"""

from __future__ import annotations

import ctypes
from dataclasses import fields
from math import prod
from pathlib import Path
from typing import Sequence

import numpy as np
import torch
from torch import Tensor

from . import _native as nat
from . import scenes
from .config import SBLConfig, fbme_profile_config
from .engine import FBMEEngine

HIDDEN = 8
TARGET_CLAMP = 20.0
WEIGHTS_DIR = Path(__file__).resolve().parent / "weights"
DEFAULT_WEIGHTS = WEIGHTS_DIR / "warm_start_256x256_128x128.npz"


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal initial parameters in the flat layout of the C ABI."""
    rng = np.random.default_rng(seed)
    parts = [
        rng.normal(0.0, np.sqrt(2.0 / 18.0), 9 * 2 * HIDDEN), np.zeros(HIDDEN),
        rng.normal(0.0, np.sqrt(2.0 / (9.0 * HIDDEN)), 9 * HIDDEN * HIDDEN), np.zeros(HIDDEN),
        0.1 * rng.normal(0.0, np.sqrt(2.0 / (9.0 * HIDDEN)), 9 * HIDDEN), np.zeros(1),
    ]
    return np.concatenate(parts).astype(np.float32)


def _ptr(t: Tensor | None) -> ctypes.c_void_p | None:
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class WarmStartNet:
    """Network parameters on a device plus the training / inference calls."""

    def __init__(self, device: torch.device, params: np.ndarray | Tensor | None = None, seed: int = 0):
        self.lib = nat.lib()
        if device.type != "cuda":
            raise RuntimeError("the warm-start network runs on CUDA devices only")
        self.device = device if device.index is not None else torch.device("cuda", torch.cuda.current_device())
        self.n_params = int(self.lib.fbme_cnn_param_count())
        p = init_params(seed) if params is None else params
        p = torch.as_tensor(p, dtype=torch.float32).to(self.device).contiguous()
        if p.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.numel()}")
        self.params = p
        self._ws: dict[tuple, tuple[Tensor, int, int]] = {}
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.step = 0

    # ---------------------------------------------------------------- io
    def save(self, path: str | Path, **meta) -> None:
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, params=self.params.cpu().numpy(), **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: str | Path, device: torch.device) -> "WarmStartNet":
        d = np.load(path)
        return cls(device, d["params"])

    # ------------------------------------------------------------- stages
    def workspace(self, batch: int, n1: int, n2: int) -> tuple[int, int]:
        key = (batch, n1, n2)
        if key not in self._ws:
            nbytes = int(self.lib.fbme_cnn_workspace_bytes(batch, n1, n2))
            if nbytes == 0:
                raise ValueError("the warm-start network needs N1 % 8 == 0 and N2 % 16 == 0")
            buf = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.device)
            self._ws[key] = (buf, (buf.data_ptr() + 255) & ~255, nbytes)
        _, ptr, nbytes = self._ws[key]
        return ptr, nbytes

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def features(self, bp: Tensor, n1: int, n2: int) -> None:
        """Features of the backprojection ``bp`` (complex64 [B, N1*N2])."""
        b = bp.shape[0]
        bp = bp.contiguous()
        ws, _ = self.workspace(b, n1, n2)
        nat.check(self.lib.fbme_cnn_features(_ptr(bp), b, n1, n2, ctypes.c_void_p(ws), self._stream()),
                  "fbme_cnn_features")

    def forward(self, batch: int, n1: int, n2: int) -> Tensor:
        out = torch.empty(batch, n1 * n2, dtype=torch.float32, device=self.device)
        ws, _ = self.workspace(batch, n1, n2)
        nat.check(self.lib.fbme_cnn_forward(_ptr(self.params), batch, n1, n2, ctypes.c_void_p(ws), _ptr(out),
                                            self._stream()), "fbme_cnn_forward")
        return out

    def backward(self, target: Tensor, batch: int, n1: int, n2: int) -> Tensor:
        """Gradient into self.grad; returns the loss as a 0-d device tensor."""
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        ws, _ = self.workspace(batch, n1, n2)
        target = target.to(torch.float32).contiguous()
        nat.check(self.lib.fbme_cnn_backward(_ptr(target), batch, n1, n2, ctypes.c_void_p(ws), _ptr(self.grad),
                                             _ptr(loss), self._stream()), "fbme_cnn_backward")
        return loss[0]

    def adam(self, lr: float) -> None:
        self.step += 1
        nat.check(self.lib.fbme_cnn_adam(_ptr(self.params), _ptr(self.grad), _ptr(self.m), _ptr(self.v),
                                         self.step, float(lr), self._stream()), "fbme_cnn_adam")

    def predict(self, bp: Tensor, n1: int, n2: int) -> Tensor:
        self.features(bp, n1, n2)
        return self.forward(bp.shape[0], n1, n2)


# ---------------------------------------------------------------- training
def plain_config(sweeps: int | None = None, profile: str = "stable") -> SBLConfig:
    """The FBME plan configuration (profiles.py:63-70, 110-115), optionally
    with a fixed sweep budget instead of the auto rule."""
    return fbme_profile_config(profile, 32, sweeps)


def training_pairs(seeds: Sequence[int], device: torch.device, *, batch: int = 64,
                   target_sweeps: int = 2, target: str = "polish") -> tuple[Tensor, Tensor]:
    """(backprojections [S, N] complex64, targets [S, N] float32) on the
    device, from plain solves.  target "polish": log(|x|^2 / (P/N) + 1e-3)
    of the plain plan's final (polished) reconstruction x, solved with the
    plan's own sweep rule; "moment": log((|mu|^2 + v) / (P/N)), the plain
    posterior second moment after ``target_sweeps`` sweeps and the final
    E-step; "prior": log(prior / (P/N)) after ``target_sweeps`` sweeps."""
    sc0 = scenes.learned_scene(int(seeds[0]))
    grid, prefix = sc0.grid, sc0.y.shape
    n = prod(grid)
    sweeps = None if target == "polish" else target_sweeps
    eng = FBMEEngine(batch, grid, prefix, plain_config(sweeps), device)
    bps, tgts = [], []
    seeds = list(seeds)
    for s0 in range(0, len(seeds), batch):
        chunk = seeds[s0:s0 + batch]
        ys = np.zeros((batch, prefix[0] * prefix[1]), np.complex64)
        for i, sd in enumerate(chunk):
            ys[i] = scenes.learned_scene(int(sd)).y.reshape(-1)
        y = torch.from_numpy(ys).to(device)
        if target == "polish":
            eng.run(y)
        else:
            eng.run_uamp(y)
        st = eng.state()
        dp = (y.abs() ** 2).mean(dim=1).clamp_min(float(np.finfo(np.float32).eps))
        if target == "polish":
            q = eng.out["x"].abs() ** 2 + 1e-3 * dp[:, None] / n
        elif target == "moment":
            q = st["mean"].abs() ** 2 + st["variance"]
        else:
            q = st["prior_variance"]
        tgt = torch.log(q.clamp_min(1e-30) / (dp[:, None] / n)).clamp(-TARGET_CLAMP, TARGET_CLAMP)
        bps.append(st["backprojection"][: len(chunk)].clone())
        tgts.append(tgt[: len(chunk)].clone())
    eng.close()
    return torch.cat(bps), torch.cat(tgts)


def train(net: WarmStartNet, bp: Tensor, target: Tensor, grid: Sequence[int], *, epochs: int = 3,
          batch: int = 16, lr: float = 2e-3, seed: int = 0, log_every: int = 200) -> list[float]:
    """Minibatch Adam on (bp, target); returns the per-step losses."""
    n1, n2 = grid
    s = bp.shape[0]
    gen = torch.Generator(device="cpu").manual_seed(seed)
    losses: list[float] = []
    total = epochs * (s // batch)
    step = 0
    for _ in range(epochs):
        order = torch.randperm(s, generator=gen)
        for b0 in range(0, s - batch + 1, batch):
            idx = order[b0:b0 + batch].to(bp.device)
            net.features(bp[idx], n1, n2)
            net.forward(batch, n1, n2)
            loss = net.backward(target[idx], batch, n1, n2)
            rate = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(total, 1)))  # cosine decay
            net.adam(rate)
            step += 1
            if step % log_every == 0 or step == total:
                losses.append(float(loss))
    return losses


# ------------------------------------------------------------ warm plans
def attach_warm_start(engine: FBMEEngine, net: WarmStartNet) -> Tensor:
    """Turn on the warm start of a native plan; returns the workspace the
    plan keeps using (hold a reference for the plan's lifetime)."""
    b = engine.batch
    shape = (nat.FbmeShape * b)(*[nat.FbmeShape(*engine.grid, *engine.sample)] * b)
    nbytes = int(net.lib.fbme_plan_warm_workspace_bytes(shape, b))
    if nbytes == 0:
        raise ValueError("the warm-start network needs N1 % 8 == 0 and N2 % 16 == 0")
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=engine.device)
    ptr = (ws.data_ptr() + 255) & ~255
    nat.check(net.lib.fbme_plan_set_warm_start(engine._plan, _ptr(net.params), ctypes.c_void_p(ptr),
                                               ctypes.c_size_t(nbytes)), "fbme_plan_set_warm_start")
    return ws


class LearnedSBLPlan:
    """Warm-started FBME plan with the plain plan as fallback, all on the device.

    One replay is two CUDA graphs on the caller's device:

    * the warm-started solve of the whole batch (the network's prior,
      ``sweeps`` UAMP sweeps, the profile's polish);
    * the fallback, on a side stream after it: the per-scene check, the
      compaction of the failing scenes into a fixed-capacity batch of
      ``fallback_capacity`` (its unused slots repeat the first failing
      scene), the plain locked solve of that batch, and the scatter of its
      rows back over the failing scenes' results.

    Nothing is read on the host.  More failures than the capacity are
    flagged on the device (``overflow``); the host re-solves the excess with
    the plain plan when the caller synchronises (``replay(synchronize=True)``,
    ``synchronize()``, or reading ``fallbacks``).

    ``pipelined=False`` (default): the caller's stream waits for the
    fallback at the end of ``replay``, so results are complete in stream
    order, as for the plain plans.  ``pipelined=True``: two warm plans take
    turns, and replay i's fallback overlaps replay i+1's warm solve; replay
    i's results are complete once the caller's stream has passed replay
    i+1 (or after ``synchronize()``), and the replay after next overwrites
    them.

    Check (per scene): finite negative log evidence, status 0, monotone
    evidence trace, and fixed-point residuals of the prior and the noise no
    larger than ``gamma_residual_max`` / ``noise_residual_max`` (above the
    90th percentiles of plain FBME-Stable solves, 0.63 and 0.006, on the
    training distribution); ``force_fallback`` marks scenes to re-solve
    regardless.
    """

    profile = "fbme-sbl-stable-learned-warm-start"

    def __init__(self, example_data: Tensor, grid_shape: Sequence[int], *, net: WarmStartNet | None = None,
                 weights: str | Path = DEFAULT_WEIGHTS, sweeps: int = 1, polish_size: int = 32,
                 warmup: int = 3, profile: str = "stable", gamma_residual_max: float = 0.75,
                 noise_residual_max: float = 0.05, fallback_capacity: int = 8,
                 pipelined: bool = False) -> None:
        from .plans import CUDAGraphSBLPlan

        if profile not in ("stable", "fast"):
            raise ValueError("profile must be 'stable' or 'fast'")
        self.net = net if net is not None else WarmStartNet.load(weights, example_data.device)
        cfg = plain_config(sweeps, profile)
        cfg.uamp_polish_size = polish_size
        self._ws: list[Tensor] = []
        self.pipelined = bool(pipelined)
        self._warm = [
            CUDAGraphSBLPlan(example_data, grid_shape, config=cfg, warmup=warmup,
                             engine_hook=lambda eng: self._ws.append(attach_warm_start(eng, self.net)))
            for _ in range(2 if self.pipelined else 1)]
        w0 = self._warm[0]
        self.device = w0.input_buffer.device
        self.batch = w0._engine.batch
        self.grid = w0._engine.grid
        self.sample = w0._engine.sample
        self.capacity = max(1, min(int(fallback_capacity), self.batch))
        plain_cfg = plain_config(None, profile)
        plain_cfg.uamp_polish_size = polish_size
        self._plain = FBMEEngine(self.capacity, self.grid, self.sample, plain_cfg, self.device)
        self._plain_in = torch.zeros(self.capacity, prod(self.sample), dtype=torch.complex64, device=self.device)
        self._plain.run(self._plain_in)  # first launches outside any capture
        self.gamma_residual_max = gamma_residual_max
        self.noise_residual_max = noise_residual_max
        self.force_fallback = torch.zeros(self.batch, dtype=torch.bool, device=self.device)
        dev = dict(device=self.device)
        self._arange_b = torch.arange(self.batch, **dev)
        self._arange_f = torch.arange(self.capacity, **dev)
        nw = len(self._warm)
        self._idxbuf = [torch.zeros(self.capacity + 1, dtype=torch.int64, **dev) for _ in range(nw)]
        self._passed = [torch.ones(self.batch, dtype=torch.bool, **dev) for _ in range(nw)]
        self._count = [torch.zeros((), dtype=torch.int64, **dev) for _ in range(nw)]
        # replays whose failures exceeded the capacity (device counter)
        self.overflows = torch.zeros((), dtype=torch.int64, **dev)
        # the fallback's short, latency-bound launches take priority over the
        # warm solve's wide grids, so they interleave instead of queueing
        self._side = torch.cuda.Stream(self.device, priority=-1)
        self._warm_done = [torch.cuda.Event() for _ in range(nw)]
        self._done = [torch.cuda.Event() for _ in range(nw)]
        self._graphs: list[torch.cuda.CUDAGraph | None] = [None] * nw
        self._graph_key: tuple | None = None
        self._slot = nw - 1
        self._pending = [False] * nw

    # ------------------------------------------------------------ results
    @property
    def result(self):
        return self._warm[self._slot].result

    @property
    def input_buffer(self) -> Tensor:
        return self._warm[(self._slot + 1) % len(self._warm)].input_buffer

    @property
    def passed(self) -> Tensor:
        """Per-scene pass flags of the last replay (device bool)."""
        return self._passed[self._slot]

    @property
    def overflow(self) -> Tensor:
        """Device flag: the last replay had more failures than the capacity."""
        return self._count[self._slot] > self.capacity

    @property
    def fallbacks(self) -> int:
        """Scenes of the last replay solved by the plain plan (synchronises)."""
        self.synchronize()
        return int(self._count[self._slot].item())

    # -------------------------------------------------------------- check
    def check(self, slot: int = 0) -> Tensor:
        """Per-scene pass flags of a warm plan's last solve (device bool)."""
        eng = self._warm[slot]._engine
        o = eng.out
        ok = torch.isfinite(o["negative_log_evidence"]) & (o["status"] == 0) & ~self.force_fallback
        if eng.native_cfg.fixed_budget_diagnostics:
            ok &= o["fixed_budget_monotone"]
            ok &= o["fixed_budget_gamma_residual"] <= self.gamma_residual_max
            ok &= o["fixed_budget_noise_residual"] <= self.noise_residual_max
        return ok

    def _fallback_body(self, s: int) -> None:
        """Check, compaction, plain re-solve and scatter of slot s (stream-ordered)."""
        F = self.capacity
        warm = self._warm[s]._engine
        ok = self.check(s)
        failed = ~ok
        count = failed.sum()
        pos = torch.cumsum(failed.to(torch.int64), 0) - 1
        target = torch.where(failed & (pos < F), pos, torch.full_like(pos, F))
        idxbuf = self._idxbuf[s]
        idxbuf.zero_()
        idxbuf.scatter_(0, target, self._arange_b)  # slot F collects the rest (discarded)
        idx = torch.where(self._arange_f < count, idxbuf[:F], idxbuf[:1].expand(F))
        flat = self._warm[s].input_buffer.reshape(self.batch, -1)
        self._plain_in.copy_(flat.index_select(0, idx))
        self._plain.run(self._plain_in)
        any_failed = count > 0
        for name, dst in warm.out.items():
            src = self._plain.out[name]
            rows = dst.index_select(0, idx)
            sel = any_failed.view(*([1] * rows.ndim))
            dst.index_copy_(0, idx, torch.where(sel, src, rows))
        self._passed[s].copy_(ok)
        self._count[s].copy_(count)
        self.overflows.add_((count > F).to(torch.int64))

    def _fallback_graph(self, s: int) -> torch.cuda.CUDAGraph:
        key = (self.gamma_residual_max, self.noise_residual_max)
        if self._graph_key != key:
            self._graphs = [None] * len(self._warm)
            self._graph_key = key
        if self._graphs[s] is None:
            torch.cuda.synchronize(self.device)
            with torch.cuda.stream(self._side):
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph, stream=self._side):
                    self._fallback_body(s)
            torch.cuda.synchronize(self.device)
            self._graphs[s] = graph
        return self._graphs[s]

    # -------------------------------------------------------------- replay
    def replay(self, data: Tensor | None = None, *, synchronize: bool = False, fallback: bool = True):
        nw = len(self._warm)
        s = (self._slot + 1) % nw
        main = torch.cuda.current_stream(self.device)
        graph = self._fallback_graph(s) if fallback else None
        if self._pending[s]:
            main.wait_event(self._done[s])  # the replay before last still fills this slot
        res = self._warm[s].replay(data, synchronize=False)
        self._slot = s
        if graph is None:
            self._pending[s] = False
            self._count[s].zero_()
            self._passed[s].copy_(self.check(s))
        else:
            self._warm_done[s].record(main)
            self._side.wait_event(self._warm_done[s])
            with torch.cuda.stream(self._side):
                graph.replay()
            self._done[s].record(self._side)
            self._pending[s] = True
            if not self.pipelined:
                main.wait_event(self._done[s])
        if synchronize:
            self.synchronize()
        return res

    def join(self) -> None:
        """Make the caller's stream wait for every pending fallback (no host
        synchronisation; failures beyond the capacity stay flagged)."""
        main = torch.cuda.current_stream(self.device)
        for s in range(len(self._warm)):
            if self._pending[s]:
                main.wait_event(self._done[s])

    def synchronize(self) -> None:
        """Wait for every replay's fallback; re-solve on the host the
        failures beyond the device capacity."""
        for s in range(len(self._warm)):
            if self._pending[s]:
                self._done[s].synchronize()
                self._pending[s] = False
                self._host_overflow(s)
        torch.cuda.synchronize(self.device)

    def _host_overflow(self, s: int) -> None:
        n = int(self._count[s].item())
        if n <= self.capacity:
            return
        bad = (~self._passed[s]).nonzero().flatten().tolist()[self.capacity:]
        warm = self._warm[s]._engine
        flat = self._warm[s].input_buffer.reshape(self.batch, -1)
        F = self.capacity
        for c0 in range(0, len(bad), F):
            grp = bad[c0:c0 + F]
            take = grp + grp[:1] * (F - len(grp))
            self._plain_in.copy_(flat[take])
            self._plain.run(self._plain_in)
            sel = torch.tensor(grp, device=self.device)
            for name, dst in warm.out.items():
                dst.index_copy_(0, sel, self._plain.out[name][: len(grp)])


def make_learned_plan(example_data: Tensor, grid_shape: Sequence[int], *, polish_size: int = 32,
                      warmup: int = 3, sweeps: int = 1, weights: str | Path = DEFAULT_WEIGHTS,
                      profile: str = "stable", pipelined: bool = False,
                      fallback_capacity: int = 8) -> LearnedSBLPlan:
    """Build the warm-started plan (same call shape as make_stable_plan)."""
    return LearnedSBLPlan(example_data, grid_shape, weights=weights, sweeps=sweeps, polish_size=polish_size,
                          warmup=warmup, profile=profile, pipelined=pipelined,
                          fallback_capacity=fallback_capacity)


def attach_warm_prior_map(engine: FBMEEngine, prior_map: Tensor | None) -> None:
    """Warm-start a native plan from the caller's own predictor: ``prior_map``
    ([B, N] float32 on the plan's device, log(prior / (P/N)) as the network
    outputs) is read at every replay until detached with None; the caller
    keeps it alive and fills it before each replay."""
    if prior_map is not None:
        if prior_map.dtype != torch.float32 or not prior_map.is_cuda or not prior_map.is_contiguous():
            raise ValueError("prior_map must be a contiguous float32 CUDA tensor")
        if tuple(prior_map.shape) != (engine.batch, engine.n_grid):
            raise ValueError(f"prior_map must have shape {(engine.batch, engine.n_grid)}")
    nat.check(engine.lib.fbme_plan_set_warm_prior_map(engine._plan, _ptr(prior_map)),
              "fbme_plan_set_warm_prior_map")
