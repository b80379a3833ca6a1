"""CUDA path against the CPU oracle, through the C-ABI (librn.so), in both
precision modes.

Tolerance: every conserved field within relative L2 1e-4 of
the oracle after N steps, each field measured against the norm of its family
(helpers.state_rel_l2). Exact mode (IEEE division/sqrt) must be much tighter:
1e-6, and bit-identical over the first steps of these cases.
"""
import numpy as np
import pytest

from helpers import assert_state_close, run_oracle

pytestmark = pytest.mark.gpu

TOL = 1e-4


def gpu_run(rn, setup, n, precision, state=None):
    g = rn.GPUSolver(setup.Nx, setup.Nr)
    g.setPrecision(precision)
    g.setGeometry(setup.geo)
    init = state if state is not None else setup.initialState()
    g.setState(init["A"], init["B"])
    if setup.injector is not None:
        rn.GPUSpray(g).resize()
        g.spray.setInjector(setup.injector)
    if n:
        g.step(n, setup.P)
    return g


def compare(rn, oracle, setup, n, precision, tol=None, identical=False):
    g = gpu_run(rn, setup, n, precision)
    o = run_oracle(oracle, setup, n)
    out, ref = g.readAll(), o.readAll()
    si_g, si_o = g.readStepInfo(), o.readStepInfo()
    g.close()
    assert np.all(np.isfinite(out["A"])) and np.all(np.isfinite(out["B"]))
    if tol is None:
        tol = TOL if precision == "fast" else 1e-6
    e = assert_state_close(out, ref, tol)
    if identical:
        assert np.array_equal(out["A"], ref["A"]) and np.array_equal(out["B"], ref["B"])
    assert abs(si_g[2] - si_o[2]) <= 1e-5 * abs(si_o[2]) + 1e-6, (si_g, si_o)
    return e


@pytest.mark.parametrize("precision", ["fast", "exact"])
@pytest.mark.parametrize("n", [1, 2, 50])
def test_plain_small_grid(rn, oracle, n, precision):
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    setup = rn.build_sim_setup(plain_small(Nx=128, Nr=48)[0])
    compare(rn, oracle, setup, n, precision, identical=precision == "exact")


@pytest.mark.parametrize("precision", ["fast", "exact"])
def test_plain_config_grid_2000_steps(rn, oracle, precision):
    """Config 1 at its full size and step count (256 x 96, 2000 steps)."""
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    cfg, steps = plain_small()
    setup = rn.build_sim_setup(cfg)
    compare(rn, oracle, setup, steps, precision, tol=TOL)


@pytest.mark.parametrize("precision", ["fast", "exact"])
@pytest.mark.parametrize("n", [1, 30])
def test_viscous_plume_small(rn, oracle, n, precision):
    from rocket_nozzle_cfd_solver_b200.configs import viscous_plume
    setup = rn.build_sim_setup(viscous_plume(Nx=128, Nr=48)[0])
    compare(rn, oracle, setup, n, precision, identical=precision == "exact")


@pytest.mark.parametrize("precision", ["fast", "exact"])
@pytest.mark.parametrize("n", [1, 30])
def test_injector_spray_small(rn, oracle, n, precision):
    from rocket_nozzle_cfd_solver_b200.configs import injector_spray
    setup = rn.build_sim_setup(injector_spray(Nx=128, Nr=48)[0])
    compare(rn, oracle, setup, n, precision)


def exit_column(state, s):
    A = np.asarray(state["A"]).reshape(s.Nr, s.Nx, 4)[:, s.iExit].ravel()
    B = np.asarray(state["B"]).reshape(s.Nr, s.Nx, 4)[:, s.iExit].ravel()
    return {"A": A, "B": B}


@pytest.mark.parametrize("case", ["config1", "viscous"])
def test_thrust_and_mass_flow_against_fp64_scheme(rn, oracle, case):
    """Exit thrust and exhaust mass flow of the FP32 CUDA path (default
    precision) within 1e-3 relative of an FP64 run of the same scheme (the
    oracle in double precision) after the same steps."""
    from rocket_nozzle_cfd_solver_b200 import configs
    if case == "config1":
        cfg, n = configs.plain_small()[0], 2000
    else:
        cfg, n = configs.viscous_plume(256, 96)[0], 2400
    s = rn.build_sim_setup(cfg)
    g = gpu_run(rn, s, n, "fast")
    gp = rn.exit_performance(s, exit_column(g.readAll(), s))
    g.close()
    op = rn.exit_performance(s, exit_column(run_oracle(oracle, s, n, fp64=True).readAll(), s))
    assert op["mdot"] > 0 and op["F"] != 0
    assert abs(gp["F"] - op["F"]) <= 1e-3 * abs(op["F"])
    assert abs(gp["mdot"] - op["mdot"]) <= 1e-3 * abs(op["mdot"])


@pytest.mark.parametrize("size", [(40, 15), (129, 47), (97, 61)])
def test_ragged_grids_bit_identical_in_exact_mode(rn, oracle, size):
    """Grids that fill no tile evenly (odd widths and heights, fewer cells
    than one row of tiles): in exact precision every tile shape gives the same
    bits, within 1e-6 of the oracle (bit-identical where pow/exp/log agree
    with the host libm) over 40 steps."""
    from rocket_nozzle_cfd_solver_b200 import solver
    from rocket_nozzle_cfd_solver_b200.configs import viscous_plume
    s = rn.build_sim_setup(viscous_plume(*size)[0])
    ref = run_oracle(oracle, s, 40).readAll()
    first = None
    for tile in solver.TILES:
        g = rn.GPUSolver(s.Nx, s.Nr)
        g.setPrecision("exact")
        g.setTile(tile)
        g.setGeometry(s.geo)
        init = s.initialState()
        g.setState(init["A"], init["B"])
        g.step(40, s.P)
        out = g.readAll()
        g.close()
        if first is None:
            first = out
            assert_state_close(out, ref, 1e-6)
        assert np.array_equal(out["A"], first["A"]) and np.array_equal(out["B"], first["B"]), tile


def test_largest_bench_grid_against_oracle(rn, oracle):
    """The 4096 x 1536 plain grid of the HBM-resident bench point (6.3 M
    cells): 15 steps against the oracle."""
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    s = rn.build_sim_setup(plain_small(4096, 1536)[0])
    compare(rn, oracle, s, 15, "fast")
