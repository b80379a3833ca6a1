"""CUDA path against the CPU oracle, through the C-ABI (librn.so).

Tolerances: float32 state, relative L2 per conserved field <= 1e-4 after N
steps (the bar for floating-point parity); one-step comparisons are tighter.
"""
import numpy as np
import pytest

from helpers import field_rel_l2, run_oracle

pytestmark = pytest.mark.gpu

TOL_N = 1e-4


def gpu_run(rn, setup, n, state=None):
    g = rn.GPUSolver(setup.Nx, setup.Nr)
    g.setGeometry(setup.geo)
    init = state if state is not None else setup.initialState()
    g.setState(init["A"], init["B"])
    if setup.injector is not None:
        rn.GPUSpray(g).resize()
        g.spray.setInjector(setup.injector)
    if n:
        g.step(n, setup.P)
    return g


def compare(rn, oracle, setup, n, tol):
    g = gpu_run(rn, setup, n)
    o = run_oracle(oracle, setup, n)
    out, ref = g.readAll(), o.readAll()
    si_g, si_o = g.readStepInfo(), o.readStepInfo()
    g.close()
    errs = {k: field_rel_l2(out[k], ref[k]) for k in ("A", "B")}
    assert np.all(np.isfinite(out["A"])) and np.all(np.isfinite(out["B"]))
    for k, e in errs.items():
        assert max(e) <= tol, f"{k}: rel L2 per field {e} > {tol}"
    assert abs(si_g[2] - si_o[2]) <= 1e-5 * abs(si_o[2]) + 1e-6, (si_g, si_o)
    return errs


@pytest.mark.parametrize("n", [1, 2, 50])
def test_plain_small_grid(rn, oracle, n):
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    cfg, _ = plain_small(Nx=128, Nr=48)
    setup = rn.build_sim_setup(cfg)
    compare(rn, oracle, setup, n, 1e-6 if n <= 2 else TOL_N)


def test_plain_config_grid_2000_steps(rn, oracle):
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    cfg, steps = plain_small()
    setup = rn.build_sim_setup(cfg)
    compare(rn, oracle, setup, steps, TOL_N)


@pytest.mark.parametrize("n", [1, 30])
def test_viscous_plume_small(rn, oracle, n):
    from rocket_nozzle_cfd_solver_b200.configs import viscous_plume
    cfg, _ = viscous_plume(Nx=128, Nr=48)
    setup = rn.build_sim_setup(cfg)
    compare(rn, oracle, setup, n, 1e-6 if n == 1 else TOL_N)


@pytest.mark.parametrize("n", [1, 30])
def test_injector_spray_small(rn, oracle, n):
    from rocket_nozzle_cfd_solver_b200.configs import injector_spray
    cfg, _ = injector_spray(Nx=128, Nr=48)
    setup = rn.build_sim_setup(cfg)
    compare(rn, oracle, setup, n, 1e-6 if n == 1 else TOL_N)
