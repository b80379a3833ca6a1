"""CPU oracle: golden fixtures, determinism, FP64 agreement and physical sanity.

The CUDA path is checked against the oracle; these tests pin the oracle. The
reference itself cannot run (WebGL2 only), so the pins are the committed
fixtures (tests/golden/make_golden.py), the reference's integer hash restated
independently in Python, and physics known answers.
"""
import math
import os

import numpy as np
import pytest

from helpers import field_rel_l2, run_oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_case(rn, name):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    return make_golden.case_setup(rn, name)


@pytest.mark.parametrize("name", ["plain", "viscous", "spray"])
def test_oracle_matches_golden(rn, oracle, name):
    s, steps = golden_case(rn, name)
    gold = np.load(os.path.join(HERE, "golden", f"oracle_{name}.npz"))
    o = run_oracle(oracle, s, steps)
    st = o.readAll()
    assert np.array_equal(st["A"].astype(np.float32), gold["A"])
    assert np.array_equal(st["B"].astype(np.float32), gold["B"])
    assert np.array_equal(o.readStepInfo().astype(np.float32), gold["stepinfo"])
    if s.injector is not None:
        par = o.readParcels()
        assert np.array_equal(par["PA"].astype(np.float32), gold["PA"])
        assert np.array_equal(par["PB"].astype(np.float32), gold["PB"])
        assert np.array_equal(o.readSrc().astype(np.float32), gold["src"])


def test_oracle_thread_count_does_not_change_bits(rn, oracle):
    s, _ = golden_case(rn, "spray")
    outs = []
    for threads in (1, 3):
        oracle.set_threads(threads)
        outs.append(run_oracle(oracle, s, 60).readAll())
    oracle.set_threads(os.cpu_count() or 1)
    assert np.array_equal(outs[0]["A"], outs[1]["A"]) and np.array_equal(outs[0]["B"], outs[1]["B"])


@pytest.mark.parametrize("name", ["plain", "viscous"])
def test_fp32_scheme_close_to_fp64(rn, oracle, name):
    s, steps = golden_case(rn, name)
    a = run_oracle(oracle, s, steps).readAll()
    b = run_oracle(oracle, s, steps, fp64=True).readAll()
    for k in ("A", "B"):
        assert max(field_rel_l2(a[k], b[k])) < 1e-3


def pcg(v):
    """The reference's 32-bit hash (spray.js:33), restated on Python integers."""
    s = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


def rnd(a, n):
    return np.float32(pcg((a + n * 7919) & 0xFFFFFFFF) & 0xFFFFFF) / np.float32(16777216.0)


def test_pcg_known_values():
    # the hash of 0 and 1 worked by hand from the shader's constants
    s0 = 2891336453
    w0 = (((s0 >> ((s0 >> 28) + 4)) ^ s0) * 277803737) & 0xFFFFFFFF
    assert pcg(0) == ((w0 >> 22) ^ w0) & 0xFFFFFFFF
    assert all(0 <= pcg(v) < 2 ** 32 for v in (1, 7919, 2654435761, 2 ** 32 - 1))


def test_spray_spawn_follows_hash(rn, oracle):
    """First step: parcels 0..3 are born from table rows chosen by the PCG hash
    with seed 1 (spray.js:46-58)."""
    s, _ = golden_case(rn, "spray")
    o = run_oracle(oracle, s, 1)
    par = o.readParcels()
    PA, PB = par["PA"].reshape(-1, 4), par["PB"].reshape(-1, 4)
    tab = s.injector["tab"].reshape(3, 256, 4)
    seed = 1
    for idx in range(4):
        pid = idx ^ ((seed * 2654435761) & 0xFFFFFFFF)
        t = int(rnd(pid, 1) * np.float32(255.999))
        assert PA[idx, 0] == tab[0, t, 0]            # x from the element
        assert PB[idx, 2] == tab[1, t, 0]            # type
        assert PB[idx, 3] == tab[2, t, 0]            # impingement x
        d = float(tab[1, t, 1]) * math.exp((float(rnd(pid, 4)) - 0.5) * 1.4)
        assert PB[idx, 0] == pytest.approx(d, rel=1e-6)
    assert np.all(PB[4:, 1] == 0)                     # nothing else alive yet
    assert o.sprayCounters() == (4, 2)


def test_quiescent_state_stays_at_rest(rn, oracle):
    """Gas at rest at ambient conditions, with the reservoir matched to the
    ambient state: the cut-cell closure balances pressure exactly in exact
    arithmetic, so only rounding-level velocities may appear."""
    from rocket_nozzle_cfd_solver_b200 import configs
    from rocket_nozzle_cfd_solver_b200.physics import R_AIR, RU, T_REF
    cfg = configs.plain_small(96, 36)[0]
    cfg.update(Tc=T_REF, Mw=RU / R_AIR, Pc=101325.0, rampMs=1e6)
    s = rn.build_sim_setup(cfg)
    N = s.Nx * s.Nr
    A = np.tile(np.array(s.P["ambCons"], dtype=np.float32), N)
    B = np.tile(np.array(s.P["ambB"], dtype=np.float32), N)
    o = run_oracle(oracle, s, 50, state={"A": A, "B": B})
    st = o.readAll()
    mask = s.mask.astype(bool)
    a = st["A"].reshape(-1, 4)[~mask]
    assert np.abs(a[:, 1:3]).max() < 1e-4
    assert np.abs(a[:, 0] - 1.0).max() < 1e-4


def test_cold_gas_thrust_near_one_d_theory(rn, oracle):
    """The plain cold-gas cone (256 x 96, 2000 steps): the exit-plane read-out
    of the oracle's state lands near 1-D nozzle theory, as the reference's
    README reports for its own solver (within a few percent)."""
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.plain_small()[0])
    o = run_oracle(oracle, s, 2000)
    st = o.readAll()
    A, B = st["A"].reshape(s.Nr, s.Nx, 4), st["B"].reshape(s.Nr, s.Nx, 4)
    perf = rn.exit_performance(s, {"A": A[:, s.iExit].reshape(-1), "B": B[:, s.iExit].reshape(-1)})
    th = s.theory
    assert perf["mdot"] == pytest.approx(th["mdot"], rel=0.05)
    assert perf["F"] == pytest.approx(th["F"], rel=0.10)
    ch = rn.cell_prim_si(s, A[0, s.iChamber], B[0, s.iChamber])
    assert abs(ch["p"] - 20e5) / 20e5 < 0.25                # the reference self-test's chamber criterion


def test_derived_restatement_on_a_uniform_state():
    """oracle/derived.py (FS_DERIVED restatement) on a uniform gas at rest and
    in motion: temperature, Mach, speed and zero vorticity / schlieren."""
    import importlib.util
    path = os.path.join(os.path.dirname(HERE), "oracle", "derived.py")
    spec = importlib.util.spec_from_file_location("oracle_derived", path)
    D = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(D)
    Nx, Nr = 6, 4
    rho, u, p, G = 1.0, 0.5, 1.0, 2.5
    A = np.tile(np.float32([rho, rho * u, 0.0, p * G + 0.5 * rho * u * u]), Nx * Nr)
    B = np.tile(np.float32([0.0, 0.0, G, 0.0]), Nx * Nr)
    mask = np.zeros(Nx * Nr, np.uint8)
    mask[0] = 1
    base = {"range": (0.0, 1.0), "RaN": 1.0, "Rs": (1.0, 1.0, 1.0), "chemV": (0, 1, 1, 0),
            "Tscale": (300.0, 3000.0, 300.0, 0.0), "schlGain": 10.0, "velScale": 100.0, "dx": 0.01}
    c = np.sqrt(1.4 * p / rho)
    out = {F: D.derived(A, B, mask, Nx, Nr, dict(base, field=F)).reshape(Nr, Nx, 4) for F in (0, 1, 2, 5, 6)}
    assert np.allclose(out[0][1:, 1:, 0], 300.0)                   # T = p/(rho R) T_REF, mapped with range (0, 1)
    assert np.allclose(out[1][1:, 1:, 0], u / c, rtol=1e-6)
    assert np.allclose(out[2][1:, 1:, 0], 0.0)
    assert np.allclose(out[5][1:, 1:, 0], u * 100.0)
    assert np.allclose(out[6][1:, 1:, 0], 0.0)
    assert np.all(out[0][0, 0] == (0, 0, 0, -1))
