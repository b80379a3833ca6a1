"""Shared helpers for the tests: setups, oracle runs and comparisons."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def field_rel_l2(a, b):
    """Relative L2 per channel of a float4 plane (ill-conditioned for a field
    that is ~0 everywhere, e.g. rho v in a flow that has not turned yet)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 4)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 4)
    return [rel_l2(a[:, c], b[:, c]) if np.linalg.norm(b[:, c]) > 0 else float(np.abs(a[:, c]).max())
            for c in range(4)]


def state_rel_l2(out, ref):
    """Relative L2 error of each conserved field against the norm of its
    family in the reference state: density and the species densities
    (rho Z, rho F, rho O) against ||rho||, each momentum component against
    ||(rho u, rho v)||, energy against ||E||, G against ||G||, and B.w (the
    inflow-speed average or rho O) against max(||B.w||, ||rho||). This is the
    tolerance metric of the parity tests (bar: 1e-4 after N steps)."""
    A, B = (np.asarray(out[k], dtype=np.float64).reshape(-1, 4) for k in ("A", "B"))
    RA, RB = (np.asarray(ref[k], dtype=np.float64).reshape(-1, 4) for k in ("A", "B"))
    n_rho = max(np.linalg.norm(RA[:, 0]), 1e-300)
    n_mom = max(np.linalg.norm(RA[:, 1:3]), 1e-300)
    n_E = max(np.linalg.norm(RA[:, 3]), 1e-300)
    n_G = max(np.linalg.norm(RB[:, 2]), 1e-300)
    n_w = max(np.linalg.norm(RB[:, 3]), n_rho)
    d = lambda x, y: float(np.linalg.norm(x - y))  # noqa: E731
    return {"rho": d(A[:, 0], RA[:, 0]) / n_rho, "rhou": d(A[:, 1], RA[:, 1]) / n_mom,
            "rhov": d(A[:, 2], RA[:, 2]) / n_mom, "E": d(A[:, 3], RA[:, 3]) / n_E,
            "rhoZ": d(B[:, 0], RB[:, 0]) / n_rho, "rhoF": d(B[:, 1], RB[:, 1]) / n_rho,
            "G": d(B[:, 2], RB[:, 2]) / n_G, "Bw": d(B[:, 3], RB[:, 3]) / n_w}


def assert_state_close(out, ref, tol):
    e = state_rel_l2(out, ref)
    bad = {k: v for k, v in e.items() if not v <= tol}
    assert not bad, f"fields above {tol}: {bad}"
    return e


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
