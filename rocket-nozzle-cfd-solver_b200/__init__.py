"""B200-native time-step hot path of the Rocket Nozzle CFD Solver.

Host side (setup, parameter block, read-outs) restates the reference's
JavaScript; the time step runs in hand-written sm_100a CUDA behind the C-ABI
library ``librn.so`` (declared in ``include/rn.h``).
"""
from . import physics, cutcell, simsetup  # noqa: F401
