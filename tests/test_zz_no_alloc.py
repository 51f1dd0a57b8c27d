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
def test_static_scratch_ragged_rows_match_workspace_topk():
    """A row length that is not a multiple of the 8192-score slice leaves a
    short last slice whose unused candidate slots feed the merge."""
    need_gpu()
    rng = np.random.default_rng(12)
    batch, n, k = 3, 8192 * 3 + 5, 32
    idx = torch.empty(batch, k, dtype=torch.int64, device="cuda")
    val = torch.empty(batch, k, dtype=torch.float32, device="cuda")
    s = rng.random((batch, n)).astype(np.float32)
    s[:, -5:] = 2.0  # the best scores sit in the short last slice
    s[1, -3] = 3.0
    scores = torch.from_numpy(s).cuda()
    ref_idx, ref_val = _topk_workspace(scores, k)
    rc, err = _topk_static(scores, k, idx, val)
    assert rc == 0, err
    torch.cuda.synchronize()
    assert torch.equal(idx, ref_idx)
    assert torch.equal(val, ref_val)


@pytest.mark.gpu
def test_static_scratch_rejects_oversize_requests():
    need_gpu()
    # 4097 rows of one slice (n <= 8192) at k = 32 need
    # 4097 * 1 * 32 * 8 = 1,048,832 bytes of candidates: 256 bytes more than
    # the 1 MiB static scratch.  The scores take 4 MiB.
    batch, n, k = 4097, 256, 32
    scores = torch.zeros(batch, n, dtype=torch.float32, device="cuda")
    idx = torch.empty(batch, k, dtype=torch.int64, device="cuda")
    val = torch.empty(batch, k, dtype=torch.float32, device="cuda")
    rc, err = _topk_static(scores, k, idx, val)
    assert rc == 1 and "static scratch" in err
    # exactly 1 MiB of candidates fits; all-equal scores take the ties path
    rc, err = _topk_static(scores[:4096], k, idx[:4096], val[:4096])
    assert rc == 0, err
    ref_idx, ref_val = _topk_workspace(scores[:4096], k)
    torch.cuda.synchronize()
    assert torch.equal(idx[:4096], ref_idx)
    assert torch.equal(ref_idx[0], torch.arange(k, device="cuda"))
    assert torch.equal(val[:4096], ref_val)
