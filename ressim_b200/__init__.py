"""B200-native fully implicit (FIM) Newton step of the ResSim black-oil simulator.

`ReservoirSimulator` mirrors the reference simulator's construction and step API; the Newton
iterations (assembly, well Schur elimination, CPR-FGMRES with block-ILU0, update and convergence
checks) run as CUDA kernels for sm_100a behind the C ABI declared in include/ressim_fim.h.
"""
import os as _os

# Every context steps on its own CUDA stream, and an ensemble drives many contexts at once.  CUDA
# maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 by default), so with more
# streams than queues the short kernels of one variant wait behind another variant's long
# pressure solve.  The value is read when the CUDA context is created, so it is set here, before
# any CUDA work, unless the caller chose one.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .deck import Deck, Well  # noqa: F401
from .simulator import ReservoirSimulator, linear_solve_bsr, linear_solve_csr  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
