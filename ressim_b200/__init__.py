"""B200-native fully implicit (FIM) Newton step of the ResSim black-oil simulator.

`ReservoirSimulator` mirrors the reference simulator's construction and step API; the Newton
iterations (assembly, well Schur elimination, CPR-FGMRES with block-ILU0, update and convergence
checks) run as CUDA kernels for sm_100a behind the C ABI declared in include/ressim_fim.h.
"""
from .deck import Deck, Well  # noqa: F401
from .simulator import ReservoirSimulator, linear_solve_bsr  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
