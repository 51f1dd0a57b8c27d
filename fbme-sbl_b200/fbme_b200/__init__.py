"""FBME-SBL plan-replay hot path on NVIDIA B200 (sm_100a).

Host layer over the C ABI of ``include/fbme_b200.h``: configuration,
result container, native engine, CUDA-Graph plans and eager solvers.  The
drop-in packages ``torch_sbl`` and ``torch_sbl_fastest_stable`` (beside this
one) re-export these under the reference's names.
"""

from .config import SBLConfig
from .result import SBLResult

__version__ = "1.1.0"
PAPER_RELEASE_ID = "FBME-SBL-TAES-v1.1"

__all__ = ["SBLConfig", "SBLResult", "PAPER_RELEASE_ID", "__version__"]
