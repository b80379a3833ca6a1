"""Shared helpers for the tests: setups, oracle runs and comparisons."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def field_rel_l2(a, b):
    """Relative L2 per conserved component (the 4 channels of a float4 plane)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 4)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 4)
    return [rel_l2(a[:, c], b[:, c]) if np.linalg.norm(b[:, c]) > 0 else float(np.abs(a[:, c]).max())
            for c in range(4)]


def run_oracle(oracle, setup, n, fp64=False, state=None):
    o = oracle.OracleSolver(setup.Nx, setup.Nr, fp64=fp64)
    o.setGeometry(setup.geo)
    init = state if state is not None else setup.initialState()
    o.setState(init["A"], init["B"])
    if setup.injector is not None:
        o.setInjector(setup.injector)
    if n:
        o.step(n, setup.P)
    return o
