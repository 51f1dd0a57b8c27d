"""Drop-in ``torch_sbl`` names backed by the B200 FBME implementation.

Mirrors the public surface of the reference package that the FBME
plan-replay path uses (torch_sbl/__init__.py of FBME-SBL v1.1): the
configuration and result types, the eager solvers and the CUDA-Graph plans.
"""

from fbme_b200 import PAPER_RELEASE_ID, __version__
from fbme_b200.config import SBLConfig
from fbme_b200.plans import (
    CUDAGraphSBLPlan,
    RealtimeSBLPlan,
    make_cuda_graph_sbl_plan,
    make_realtime_sbl_plan,
)
from fbme_b200.result import SBLResult
from fbme_b200.solver import clear_operator_cache, fast_sbl, sbl_1d, sbl_2d

__all__ = [
    "PAPER_RELEASE_ID", "__version__", "SBLConfig", "SBLResult", "clear_operator_cache",
    "fast_sbl", "sbl_1d", "sbl_2d", "CUDAGraphSBLPlan", "RealtimeSBLPlan",
    "make_cuda_graph_sbl_plan", "make_realtime_sbl_plan",
]
