"""Helpers shared by the GPU tests."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")


def rel_l2(a, b) -> float:
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# Parity tolerances (fixed by the task): x within 1e-4 relative L2 of the
# reference, identical support, posterior variance within 1e-3 relative.
X_TOL = 1e-4
PV_TOL = 1e-3
