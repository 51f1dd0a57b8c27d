"""Failure detection on the GPU without a fault: a bounded device wait that
runs out.

fbme_selftest_stage_timeout launches one DFT stage tile whose operand
producer is held back (it issues no load, copy or arrive), so the
tensor-core issuer and the epilogue wait for data that never comes.  With a
short wait limit (2e6 SM cycles, about a millisecond) both waits run out;
the kernel must record FBME_STATUS_TIMEOUT, free its tensor memory and
return, and the context must stay usable for the next solve.
"""

import ctypes
import time

import pytest

from gpu_util import need_gpu

torch = pytest.importorskip("torch")


@pytest.mark.gpu
def test_stage_wait_runs_out_records_timeout_and_returns():
    need_gpu()
    from fbme_b200 import _native as nat

    lib = nat.lib()
    nbytes = int(lib.fbme_selftest_workspace_bytes())
    ws = torch.zeros(nbytes + 256, dtype=torch.uint8, device="cuda")
    ptr = (ws.data_ptr() + 255) & ~255
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = lib.fbme_selftest_stage_timeout(ctypes.c_void_p(ptr), ctypes.c_size_t(nbytes),
                                         ctypes.c_void_p(status.data_ptr()), 2_000_000, stream)
    nat.check(rc, "fbme_selftest_stage_timeout")
    torch.cuda.synchronize()  # the kernel returned
    dt = time.perf_counter() - t0
    assert int(status.item()) & nat.STATUS_TIMEOUT
    assert dt < 5.0, dt
    assert int(ws.count_nonzero()) == 0  # nothing was read into or written to the tile buffers

    # the context is intact: a plan solves a scene correctly afterwards
    from fbme_b200 import scenes
    from oracle import fbme_oracle as O
    from torch_sbl_fastest_stable import make_stable_plan

    sc = scenes.config_scene("c1", 0)
    y = torch.from_numpy(sc.y).cuda()
    res = make_stable_plan(y, sc.grid, warmup=1).replay(y, synchronize=True)
    assert int(res.status.item()) == 0
    ref = O.fbme_solve(sc.y, sc.grid, "stable")
    x, xr = res.x.cpu().numpy().reshape(-1), ref["x"].reshape(-1)
    assert set(x.nonzero()[0]) == set(xr.nonzero()[0])
