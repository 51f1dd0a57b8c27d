"""Allocation-free top-k (fbme_topk_static) against the workspace version.

Some callers cannot allocate device memory when they need a top-k (code
running inside another component's CUDA-graph capture, real-time hosts with
a frozen memory budget, FFI hosts that only get device pointers), so the
library offers one entry point whose scratch is a static device array.  This
test calls it through the C ABI twice in a row, on different inputs, and
checks that each call returns exactly what fbme_topk returns (index work:
bit-exact).  It runs last (file name) and also passes alone.
"""

import ctypes

import numpy as np
import pytest

from gpu_util import need_gpu

torch = pytest.importorskip("torch")


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _topk_workspace(scores, k):
    from fbme_b200 import _native as nat

    lib = nat.lib()
    batch, n = scores.shape
    nbytes = lib.fbme_topk_workspace_bytes(n, k, batch)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    idx = torch.empty(batch, k, dtype=torch.int64, device="cuda")
    val = torch.empty(batch, k, dtype=torch.float32, device="cuda")
    rc = lib.fbme_topk(ctypes.c_void_p(scores.data_ptr()), n, k, batch, ctypes.c_void_p(ws.data_ptr()),
                       ctypes.c_size_t(nbytes), ctypes.c_void_p(idx.data_ptr()),
                       ctypes.c_void_p(val.data_ptr()), _stream())
    nat.check(rc, "fbme_topk")
    return idx, val


def _topk_static(scores, k, idx, val):
    from fbme_b200 import _native as nat

    lib = nat.lib()
    batch, n = scores.shape
    rc = lib.fbme_topk_static(ctypes.c_void_p(scores.data_ptr()), n, k, batch,
                              ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(val.data_ptr()), _stream())
    return rc, lib.fbme_topk_static_error().decode()


@pytest.mark.gpu
def test_static_scratch_topk_matches_workspace_topk_twice():
    need_gpu()
    rng = np.random.default_rng(11)
    batch, n, k = 4, 65536, 32
    # outputs allocated up front; the entry point itself allocates nothing
    idx = torch.empty(batch, k, dtype=torch.int64, device="cuda")
    val = torch.empty(batch, k, dtype=torch.float32, device="cuda")
    for call in range(2):
        s = rng.random((batch, n)).astype(np.float32)
        s[:, 17:4000:13] = s.max() * 0.999  # ties straddling the cut
        scores = torch.from_numpy(s).cuda()
        ref_idx, ref_val = _topk_workspace(scores, k)
        rc, err = _topk_static(scores, k, idx, val)
        assert rc == 0, err
        torch.cuda.synchronize()
        assert torch.equal(idx, ref_idx), f"call {call}"
        assert torch.equal(val, ref_val), f"call {call}"


@pytest.mark.gpu
def test_static_scratch_rejects_oversize_requests():
    need_gpu()
    batch, n, k = 64, 262144, 32  # needs 64 * 32 * 32 * 8 = 512 KiB... scale past 1 MiB
    scores = torch.zeros(batch * 4, n, dtype=torch.float32, device="cuda")
    idx = torch.empty(batch * 4, k, dtype=torch.int64, device="cuda")
    val = torch.empty(batch * 4, k, dtype=torch.float32, device="cuda")
    rc, err = _topk_static(scores, k, idx, val)
    assert rc == 1 and "static scratch" in err
