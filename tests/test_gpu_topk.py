"""Stage entry point fbme_topk (C ABI) against a stable descending sort:
the k largest scores, largest first, ties by lower index (torch.topk at
torch_sbl/solver.py:1931)."""

import ctypes

import numpy as np
import pytest

from gpu_util import need_gpu

torch = pytest.importorskip("torch")


def topk_native(scores: "torch.Tensor", k: int):
    from fbme_b200 import _native as nat

    lib = nat.lib()
    batch, n = scores.shape
    nbytes = lib.fbme_topk_workspace_bytes(n, k, batch)
    assert nbytes > 0, nat.last_error()
    ws = torch.empty(nbytes, dtype=torch.uint8, device=scores.device)
    idx = torch.empty(batch, k, dtype=torch.int64, device=scores.device)
    val = torch.empty(batch, k, dtype=torch.float32, device=scores.device)
    rc = lib.fbme_topk(ctypes.c_void_p(scores.data_ptr()), n, k, batch,
                       ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(nbytes),
                       ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(val.data_ptr()),
                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    nat.check(rc, "fbme_topk")
    return idx, val


def reference_topk(s: np.ndarray, k: int):
    order = np.argsort(-s, axis=1, kind="stable")[:, :k]
    return order, np.take_along_axis(s, order, axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,batch", [(65536, 32, 3), (8192 * 3 + 17, 12, 2), (40, 32, 1), (262144, 32, 1)])
def test_topk_matches_stable_sort(n, k, batch):
    need_gpu()
    rng = np.random.default_rng(n + k)
    s = rng.random((batch, n)).astype(np.float32) * 10
    s[:, 5:200:7] = 3.25  # ties, some near the threshold
    s[0, min(100, n - 1)] = 9.9999990
    idx, val = topk_native(torch.from_numpy(s).cuda(), k)
    ri, rv = reference_topk(s, k)
    np.testing.assert_array_equal(idx.cpu().numpy(), ri)
    np.testing.assert_array_equal(val.cpu().numpy(), rv)


@pytest.mark.gpu
def test_topk_all_ties_takes_lowest_indices():
    need_gpu()
    s = np.full((2, 20000), 1.5, np.float32)
    idx, _ = topk_native(torch.from_numpy(s).cuda(), 32)
    assert np.array_equal(idx.cpu().numpy()[0], np.arange(32))


def _check(s: np.ndarray, k: int):
    idx, val = topk_native(torch.from_numpy(s).cuda(), k)
    ri, rv = reference_topk(s, k)
    np.testing.assert_array_equal(idx.cpu().numpy(), ri)
    np.testing.assert_array_equal(val.cpu().numpy(), rv)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 2, 7, 16, 31, 32])
def test_topk_every_k_ragged_n(k):
    """A slice's k best are found among the keys at or above the k-th largest
    thread maximum; the last slice is ragged."""
    need_gpu()
    rng = np.random.default_rng(100 + k)
    _check((rng.standard_normal((3, 8192 * 2 + 4099)) * 3).astype(np.float32), k)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["few_levels", "one_thread_peaks", "inf_and_sparse", "tiny_n"])
def test_topk_adversarial_keys(kind):
    """Ties crowding the threshold (the candidate list overflows and the radix
    select over all keys decides), the best keys all held by one thread,
    infinities among sparse peaks, and fewer entries than threads."""
    need_gpu()
    rng = np.random.default_rng(7)
    if kind == "few_levels":
        s = rng.integers(0, 4, (2, 65536)).astype(np.float32)
    elif kind == "one_thread_peaks":
        s = rng.random((2, 65536)).astype(np.float32)
        s[:, 3::256][:, :40] += 10.0  # slice 0, thread 3: 32 keys; slice 1: 8 more
    elif kind == "inf_and_sparse":
        s = np.zeros((2, 50000), np.float32)
        s[:, rng.choice(50000, 9, replace=False)] = rng.random(9).astype(np.float32) + 1
        s[0, 17] = np.inf
        s[1, 4000:4100] = -np.inf
        s[1, 33] = np.inf
    else:
        s = rng.random((4, 20)).astype(np.float32)
        s[:, 3] = s[:, 5]
    _check(s, min(32, s.shape[1]))
