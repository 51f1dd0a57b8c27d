"""Host logic of the mode="cg" path (no GPU): probe budget, probe streams,
configuration mapping and the supported-feature checks."""

import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

from fbme_b200 import _native as nat
from fbme_b200.cg import check_cg_supported, make_probes, probe_count, resolve_cg_config
from fbme_b200.config import SBLConfig
from oracle import fbme_oracle as O

PROBES = Path(__file__).parent / "golden" / "cg" / "probes.npz"


@pytest.mark.parametrize("grid,sample,expected", [
    ((64, 64), (32, 32), 32),       # N/M = 4: 8*2 = 16 -> hutchinson_probes
    ((256, 256), (128, 128), 32),
    ((512, 512), (64, 64), 128),    # N/M = 64 > 16: max(64, 128) capped at 128
    ((512, 512), (128, 128), 32),   # N/M = 16: 8*4 = 32
    ((300, 300), (60, 60), 50),     # N/M = 25: max(40, 50)
])
def test_probe_budget_follows_reference(grid, sample, expected):
    cfg = SBLConfig()
    n, m = int(np.prod(grid)), int(np.prod(sample))
    assert probe_count(cfg, n, m) == expected
    assert O.cg_probe_count(O.OracleConfig(), n, m) == expected


def test_probe_streams_match_reference_generator():
    g = np.load(PROBES)
    cpu = torch.device("cpu")
    z = make_probes(2, 32 * 24, 8, device=cpu, seed=5)
    np.testing.assert_array_equal(z.numpy().astype(np.int8), g["rademacher_8"])
    np.testing.assert_array_equal(O.rademacher_probes(2, 32 * 24, 8, 5).astype(np.int8),
                                  g["rademacher_8"])
    for count in (8, 13, 32):
        z = make_probes(2, 32 * 24, count, device=cpu, seed=5, probe_type="hadamard",
                        sample_shape=(32, 24))
        np.testing.assert_array_equal(z.numpy().astype(np.int8), g[f"hadamard_{count}"])


def test_cg_schedule_matches_oracle():
    cfg = SBLConfig(adaptive_probes=True)
    ocfg = O.OracleConfig(adaptive_probes=True)
    nc = resolve_cg_config(cfg, 4096, 1024)
    for it in (1, 5, 6, 15, 16, 40):
        cnt, tol = O.cg_schedule(it, ocfg, nc.probes)
        assert 1 <= cnt <= nc.probes
        assert tol >= cfg.cg_tolerance
    assert O.cg_schedule(3, ocfg, 32)[0] == 16
    assert O.cg_schedule(10, ocfg, 32)[0] == 24
    assert O.cg_schedule(20, ocfg, 32)[0] == 32


def test_resolve_cg_config_fields():
    cfg = SBLConfig(mode="cg", max_iter=77, cg_max_iter=90, cg_check_interval=5, seed=3,
                    noise_update="evidence", fixed_noise_variance=0.25, initialization="uniform")
    c = resolve_cg_config(cfg, 65536, 16384)
    assert (c.max_iter, c.cg_max_iter, c.cg_check_interval) == (77, 90, 5)
    assert c.noise_update == 1 and c.fixed_noise_variance == pytest.approx(0.25)
    assert c.initialization_blend < 0 and c.probes == 32 and c.preconditioner_rank == 32
    assert c.dft_terms == cfg.cg_dft_terms
    lib = nat.lib()
    shape = nat.FbmeShape(256, 256, 128, 128)
    assert lib.fbme_cg_workspace_bytes(ctypes.byref(shape), 2, ctypes.byref(c)) > 2 * 33 * 16384 * 8
    bad = nat.FbmeShape(64, 64, 65, 32)
    assert lib.fbme_cg_workspace_bytes(ctypes.byref(bad), 1, ctypes.byref(c)) == 0
    plan = ctypes.c_void_p()
    rc = lib.fbme_cg_create(ctypes.byref(bad), 1, ctypes.byref(c), None, 0, None, ctypes.byref(plan))
    assert rc == nat.FBME_ERR_INVALID


def test_unsupported_cg_features_raise():
    check_cg_supported(SBLConfig(), batch=1)  # the single-scene active-set switch is built
    with pytest.raises(NotImplementedError, match="active_set_max_size"):
        check_cg_supported(SBLConfig(active_set_max_size=2048), batch=1)
    check_cg_supported(SBLConfig(active_set_max_size=2048), batch=2)  # batches never switch
    check_cg_supported(SBLConfig(), batch=2)
    check_cg_supported(SBLConfig(active_set=False), batch=1)
    with pytest.raises(NotImplementedError, match="circulant"):
        check_cg_supported(SBLConfig(cg_preconditioner="circulant", active_set=False), batch=1)
    with pytest.raises(NotImplementedError, match="joint_sparsity"):
        check_cg_supported(SBLConfig(joint_sparsity=True), batch=2)
