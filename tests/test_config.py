"""SBLConfig mirror: presets, validation errors, and the resolution of the
hot-path fields into the C ABI's FbmeConfig."""

import pytest

from fbme_b200.config import SBLConfig
from fbme_b200.engine import resolve_native_config, uamp_iteration_limit


def test_paper_preset_values():
    c = SBLConfig.paper_hybrid_uamp()
    assert c.mode == "uamp" and c.tol == 0.0 and c.damping == 0.15
    assert c.uamp_damping == 0.05 and not c.uamp_adaptive_damping
    assert c.uamp_iteration_scale == 0.8 and c.uamp_iteration_offset == 0.0 and c.uamp_min_iter == 3
    assert c.uamp_polish_size == 32 and c.uamp_polish_iterations == 3
    assert c.uamp_polish_residual_exchange_size == 12 and c.uamp_polish_evidence_margin_factor == 64.0
    assert c.uamp_polish_prune_tail and c.uamp_polish_reinitialize and c.uamp_polish_evidence_gate
    assert c.uamp_support_false_alarm_budget == 0.5 and c.uamp_polish_fixed_budget_diagnostics
    assert (c.hyper_shape, c.hyper_rate, c.noise_shape, c.noise_rate) == (0.0, 0.0, 0.0, 0.0)
    assert c.uamp_backend == "triton" and not c.return_history
    assert SBLConfig.realtime_hybrid_uamp() == c
    c.validate()


def test_fast_presets():
    h = SBLConfig.fast_hybrid_uamp()
    assert h.uamp_iteration_offset == 1.0 and h.uamp_iteration_scale == 1.0
    assert h.uamp_polish_iterations == 2 and h.uamp_polish_residual_exchange_size == 0
    u = SBLConfig.fast_uamp()
    assert u.mode == "uamp" and u.uamp_polish_size == 32 and not u.active_set
    t = SBLConfig.taes_hybrid_uamp()
    assert t.uamp_polish_iterations == 8 and t.uamp_polish_high_precision


@pytest.mark.parametrize("kw,msg", [
    (dict(damping=1.0), "damping must satisfy"),
    (dict(mode="fft"), "mode must be"),
    (dict(uamp_polish_residual_exchange_size=40), "exchange_size must be in"),
    (dict(uamp_polish_residual_exchange_size=4, uamp_polish_iterations=1), "Residual support exchange"),
    (dict(uamp_polish_support_repairs=1), "requires uamp_polish_global_certificate"),
    (dict(uamp_polish_fixed_budget_diagnostics=True), "fixed_budget_diagnostics requires"),
    (dict(cg_fixed_iterations=200), "cannot exceed cg_max_iter"),
])
def test_validation_errors(kw, msg):
    with pytest.raises(ValueError, match=msg):
        SBLConfig(**kw).validate()


def test_uamp_budget_and_native_mapping():
    stable = SBLConfig.paper_hybrid_uamp(uamp_polish_size=32)
    # T_u = min(max_iter, max(max(min_iter, uamp_min_iter), ceil(0.8 N/M)))
    assert uamp_iteration_limit(stable, 65536, 16384) == 4
    assert uamp_iteration_limit(stable, 512 * 512, 256 * 192) == 5
    assert uamp_iteration_limit(stable, 1280, 320) == 4
    assert uamp_iteration_limit(stable, 4096, 1024) == 4
    n = resolve_native_config(stable, (256, 256), (128, 128))
    assert n.uamp_iterations == 4 and n.polish_size == 32 and n.exchange_size == 12
    assert abs(n.uamp_damping - 0.05) < 1e-7 and n.fixed_budget_diagnostics == 1
    assert abs(n.support_false_alarm_budget - 0.5) < 1e-7
    # automatic DFT form: FP32 FFT stages where both grid lengths are 2^a or
    # 3 * 2^a (<= 512) in an equal-shape plan, else the 3-term products
    assert n.dft_terms == 0
    assert resolve_native_config(stable, (40, 32), (20, 16)).dft_terms == 3
    assert resolve_native_config(stable, (384, 192), (100, 90)).dft_terms == 0
    assert resolve_native_config(stable, (1024, 256), (512, 128)).dft_terms == 3
    assert resolve_native_config(stable, (256, 256), (128, 128), uneven=True).dft_terms == 3
    # an uneven plan runs one form for all its buckets: the FFT stages when
    # every grid allows them
    from fbme_b200.engine import resolve_uneven_dft_terms

    assert resolve_uneven_dft_terms(-1, [(256, 256), (192, 256), (384, 256), (128, 128)]) == 0
    assert resolve_uneven_dft_terms(-1, [(256, 256), (40, 32)]) == 3
    assert resolve_uneven_dft_terms(3, [(256, 256)]) == 3
    assert resolve_native_config(SBLConfig.paper_hybrid_uamp(uamp_polish_size=32, dft_terms=6),
                                 (256, 256), (128, 128)).dft_terms == 6
    hybrid = SBLConfig.fast_hybrid_uamp()
    h = resolve_native_config(hybrid, (256, 256), (128, 128))
    # adaptive damping: max(0.1, min(0.8, 0.02 * N / M)) = 0.1
    assert abs(h.uamp_damping - 0.1) < 1e-7 and h.uamp_iterations == 5
    small = resolve_native_config(stable, (6, 6), (3, 3))
    assert small.polish_size == 32 or small.polish_size == 36
    tiny = SBLConfig.paper_hybrid_uamp(uamp_polish_size=32)
    t = resolve_native_config(tiny, (8, 5), (4, 2))
    assert t.polish_size == 32 and t.exchange_size == min(12, 31, 40 - 32)
