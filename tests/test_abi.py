"""The C-ABI library loads and exports every symbol include/*.h declares;
host-side validation returns the documented codes without touching a GPU."""

import ctypes
import re
from pathlib import Path

import pytest

from fbme_b200 import _native as nat

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def _declared():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(fbme_[a-z0-9_]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported_and_bound():
    lib = nat.lib()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert declared <= set(nat.SIGNATURES), declared - set(nat.SIGNATURES)


def test_version_and_group_names():
    lib = nat.lib()
    assert b"sm_100a" in lib.fbme_version()
    names = [lib.fbme_profile_group_name(g).decode() for g in range(nat.NUM_GROUPS)]
    assert names[2] == "adjoint_denoise" and all(names)


def _cfg(**kw):
    from fbme_b200.config import SBLConfig
    from fbme_b200.engine import resolve_native_config

    cfg = SBLConfig.paper_hybrid_uamp(uamp_polish_size=32, **kw)
    return resolve_native_config(cfg, (256, 256), (128, 128))


def test_workspace_bytes_and_validation_codes():
    lib = nat.lib()
    c = _cfg()
    shapes = (nat.FbmeShape * 2)(nat.FbmeShape(256, 256, 128, 128), nat.FbmeShape(256, 256, 128, 128))
    nbytes = lib.fbme_plan_workspace_bytes(shapes, 2, ctypes.byref(c))
    assert nbytes > 2 * 256 * 256 * 8
    bad = (nat.FbmeShape * 1)(nat.FbmeShape(64, 64, 128, 32))
    assert lib.fbme_plan_workspace_bytes(bad, 1, ctypes.byref(c)) == 0
    plan = ctypes.c_void_p()
    rc = lib.fbme_plan_create(bad, 1, ctypes.byref(c), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_INVALID and "0 < M <= N" in nat.last_error()
    # scenes of different shapes make an uneven plan: sized, then refused
    # here only for the missing workspace, with the FP32 FFT stages (what
    # the 256x256 config resolves to) or the tensor-core stages; the FFT
    # stages need every grid length to allow them
    assert c.dft_terms == 0
    uneven = (nat.FbmeShape * 2)(nat.FbmeShape(64, 64, 32, 32), nat.FbmeShape(128, 64, 32, 32))
    assert lib.fbme_plan_workspace_bytes(uneven, 2, ctypes.byref(c)) > 0
    rc = lib.fbme_plan_create(uneven, 2, ctypes.byref(c), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_WORKSPACE
    odd = (nat.FbmeShape * 2)(nat.FbmeShape(64, 64, 32, 32), nat.FbmeShape(40, 64, 32, 32))
    assert lib.fbme_plan_workspace_bytes(odd, 2, ctypes.byref(c)) == 0
    c3 = _cfg(dft_terms=3)
    assert lib.fbme_plan_workspace_bytes(uneven, 2, ctypes.byref(c3)) > 0
    rc = lib.fbme_plan_create(uneven, 2, ctypes.byref(c3), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_WORKSPACE
    rc = lib.fbme_plan_create(shapes, 2, ctypes.byref(c), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_WORKSPACE
    big = _cfg()
    big.polish_size = 64
    rc = lib.fbme_plan_create(shapes, 2, ctypes.byref(big), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        nat.check(nat.FBME_ERR_INVALID, "x")
    with pytest.raises(NotImplementedError):
        nat.check(nat.FBME_ERR_UNSUPPORTED, "x")
    with pytest.raises(RuntimeError):
        nat.check(nat.FBME_ERR_CUDA, "x")


def test_batch_limits_are_rejected_on_the_host():
    """Launches put a plan's scenes and top-k rows on a 65535-limited grid
    dimension; larger requests fail at validation with a clear code."""
    lib = nat.lib()
    c = _cfg()
    c.exchange_size = 12
    n = 65536
    shapes = (nat.FbmeShape * n)(*([nat.FbmeShape(64, 64, 32, 32)] * n))
    assert lib.fbme_plan_workspace_bytes(shapes, n, ctypes.byref(c)) == 0
    plan = ctypes.c_void_p()
    rc = lib.fbme_plan_create(shapes, n, ctypes.byref(c), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_UNSUPPORTED and "65535" in nat.last_error()
    ok = lib.fbme_plan_workspace_bytes(shapes, n - 1, ctypes.byref(c))
    assert ok > 0
    assert lib.fbme_topk_workspace_bytes(100, 1, 65536) == 0
    assert lib.fbme_topk_workspace_bytes(100, 1, 65535) > 0
    # non-NULL stand-ins: the size check fails before any pointer is used
    fake = ctypes.c_void_p(256)
    rc = lib.fbme_topk(fake, 100, 1, 65536, fake, 0, fake, fake, None)
    assert rc == nat.FBME_ERR_INVALID and "65535" in nat.last_error()


def test_selftest_arguments_are_checked_on_the_host():
    lib = nat.lib()
    n = lib.fbme_selftest_workspace_bytes()
    assert n > 0
    fake = ctypes.c_void_p(256)
    assert lib.fbme_selftest_stage_timeout(fake, n, fake, 10, None) == nat.FBME_ERR_INVALID
    assert lib.fbme_selftest_stage_timeout(ctypes.c_void_p(257), n, fake, 10**6, None) == nat.FBME_ERR_WORKSPACE
    assert lib.fbme_selftest_stage_timeout(fake, n - 1, fake, 10**6, None) == nat.FBME_ERR_WORKSPACE
    assert lib.fbme_selftest_stage_timeout(None, n, fake, 10**6, None) == nat.FBME_ERR_INVALID
