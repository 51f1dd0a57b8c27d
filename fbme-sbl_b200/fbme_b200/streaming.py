"""Host-resident batches through a captured plan, transfers overlapped.

A plan replay reads its observations from device memory and leaves its
results there.  ``HostPipeline`` feeds a plan from pinned host batches and
returns each batch's result to pinned host buffers, with both copies
overlapped with the solves of neighbouring batches:

    h2d stream      H2D y[i+1] -> stage_in[(i+1) % 2]
    compute stream  stage_in[i % 2] -> plan input; replay; result -> stage_out[i % 2]
    d2h stream      stage_out[i % 2] -> host result i

so a step costs max(solve, H2D, D2H) instead of their sum.  Two staging
slots decouple the streams; events order every reuse of a slot.

Results come back compact by default: the plans' x is exactly zero off
the active set, so the active indices and their x values
(``FbmeOutputs.active_indices`` / ``active_values``) are the whole
reconstruction, together with the noise variance, the negative log
evidence and the status word.  ``dense=True`` returns the dense x instead.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch
from torch import Tensor


@dataclass
class HostResult:
    """Pinned host buffers of one batch's result."""

    noise_variance: Tensor
    negative_log_evidence: Tensor
    status: Tensor
    active_indices: Tensor | None = None  # [B, K] int64 (compact)
    active_values: Tensor | None = None   # [B, K] complex64 (compact)
    x: Tensor | None = None               # [B, N1, N2] complex64 (dense)

    def dense_x(self, grid) -> Tensor:
        """The dense reconstruction on the host (from the compact form)."""
        if self.x is not None:
            return self.x
        b = self.active_indices.shape[0]
        x = torch.zeros(b, grid[0] * grid[1], dtype=torch.complex64)
        x.scatter_(1, self.active_indices, self.active_values)
        return x.view(b, *grid)


class HostPipeline:
    """Solve a stream of pinned host batches with a fixed-shape plan.

    ``plan`` is a captured plan (``make_stable_plan`` / ``make_fastest_plan``
    / ``CUDAGraphSBLPlan``) whose input shape every batch has.  ``submit``
    enqueues one batch and returns at once; a batch's ``HostResult`` is
    complete after ``wait(result)`` or ``synchronize()``.
    """

    def __init__(self, plan, *, dense: bool = False) -> None:
        self.plan = plan
        self.dense = dense
        eng = plan._engine
        self.device = plan.device
        self._out = eng.out
        self.batch = eng.batch
        self.grid = eng.grid
        self.K = int(eng.native_cfg.polish_size)
        dev = self.device
        self._in = [torch.empty_like(plan.input_buffer) for _ in range(2)]
        B, K = self.batch, self.K
        self._stage = []
        for _ in range(2):
            st = {"noise_variance": torch.empty(B, dtype=torch.float32, device=dev),
                  "negative_log_evidence": torch.empty(B, dtype=torch.float32, device=dev),
                  "status": torch.empty(B, dtype=torch.int32, device=dev)}
            if dense:
                st["x"] = torch.empty(B, *self.grid, dtype=torch.complex64, device=dev)
            else:
                st["active_indices"] = torch.empty(B, K, dtype=torch.int64, device=dev)
                st["active_values"] = torch.empty(B, K, dtype=torch.complex64, device=dev)
            self._stage.append(st)
        self.h2d = torch.cuda.Stream(device=dev)
        self.d2h = torch.cuda.Stream(device=dev)
        ev = lambda: torch.cuda.Event()  # noqa: E731
        self._in_ready = [ev(), ev()]    # H2D into slot done
        self._in_free = [ev(), ev()]     # slot copied into the plan input
        self._out_ready = [ev(), ev()]   # results copied into the slot
        self._out_free = [ev(), ev()]    # slot copied to the host
        self._used = [False, False]
        self._step = 0

    def host_result(self) -> HostResult:
        """Pinned host buffers for one batch's result."""
        B, K = self.batch, self.K
        pin = dict(pin_memory=True)
        r = HostResult(torch.empty(B, dtype=torch.float32, **pin),
                       torch.empty(B, dtype=torch.float32, **pin),
                       torch.empty(B, dtype=torch.int32, **pin))
        if self.dense:
            r.x = torch.empty(B, *self.grid, dtype=torch.complex64, **pin)
        else:
            r.active_indices = torch.empty(B, K, dtype=torch.int64, **pin)
            r.active_values = torch.empty(B, K, dtype=torch.complex64, **pin)
        return r

    def submit(self, y_host: Tensor, result: HostResult) -> None:
        """Enqueue one batch: pinned ``y_host`` (the plan's input shape) to
        the device, one replay, the result to ``result``."""
        if tuple(y_host.shape) != tuple(self.plan.input_buffer.shape) or y_host.dtype != torch.complex64:
            raise ValueError(f"expected complex64 host data of shape {tuple(self.plan.input_buffer.shape)}")
        slot = self._step % 2
        comp = torch.cuda.current_stream(self.device)
        # H2D into the slot once the batch two steps back has left it
        if self._step == 0:
            self.h2d.wait_stream(comp)
        if self._used[slot]:
            self.h2d.wait_event(self._in_free[slot])
        with torch.cuda.stream(self.h2d):
            self._in[slot].copy_(y_host, non_blocking=True)
            self._in_ready[slot].record(self.h2d)
        # solve, then copy the result into the slot once the host copy of
        # the batch two steps back has left it
        comp.wait_event(self._in_ready[slot])
        self.plan.input_buffer.copy_(self._in[slot])
        self._in_free[slot].record(comp)
        self.plan.replay()
        if self._used[slot]:
            comp.wait_event(self._out_free[slot])
        st = self._stage[slot]
        for name, t in st.items():
            src = self._out[name]
            t.copy_(src.view(t.shape))
        self._out_ready[slot].record(comp)
        # D2H of the slot
        self.d2h.wait_event(self._out_ready[slot])
        with torch.cuda.stream(self.d2h):
            for name, t in st.items():
                getattr(result, name).copy_(t, non_blocking=True)
            self._out_free[slot].record(self.d2h)
        result._done = self._out_free[slot]
        self._used[slot] = True
        self._step += 1

    def wait(self, result: HostResult) -> HostResult:
        """Block the host until ``result`` is complete."""
        ev = getattr(result, "_done", None)
        if ev is not None:
            ev.synchronize()
        return result

    def join(self) -> None:
        """Make the current stream wait for every copy enqueued so far
        (device-side; for timing with events on the current stream)."""
        comp = torch.cuda.current_stream(self.device)
        comp.wait_stream(self.h2d)
        comp.wait_stream(self.d2h)

    def synchronize(self) -> None:
        self.join()
        torch.cuda.synchronize(self.device)
