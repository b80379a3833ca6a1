"""B200-native time-step hot path of the Rocket Nozzle CFD Solver.

Host side (setup, parameter block, read-outs) restates the reference's
JavaScript; the time step runs in hand-written sm_100a CUDA behind the C-ABI
library ``librn.so`` (declared in ``include/rn.h``). ``GPUSolver`` and
``GPUSpray`` mirror the reference's solver classes over that library.
"""
from . import physics, cutcell, simsetup  # noqa: F401
from .simsetup import build_sim_setup, compute_params, exit_performance, cell_prim_si  # noqa: F401
from .solver import GPUSolver, GPUSpray, SolverBatch, SolveServer, RnError, params_from_P  # noqa: F401
