"""Device read-outs against the host restatement of the reference's
JavaScript read-outs, on the same device state: the flow-separation point
(wallSeparation, simsetup.js:352-373, restated in simsetup.wall_separation
over the read-back wall row)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def viscous(rn, Nx=256, Nr=96, alt_km=0.0):
    from rocket_nozzle_cfd_solver_b200 import configs
    return rn.build_sim_setup(configs.viscous_plume(Nx, Nr, alt_km)[0])


def host_separation(rn, g, s, paSi):
    from rocket_nozzle_cfd_solver_b200 import simsetup
    tex = g.drawWallRow()
    row = g._readRect(tex, 0, 0, s.Nx, 1)
    return simsetup.wall_separation(s, row, paSi)


def assert_same(dev, host):
    if host is None:
        assert dev is None
        return
    assert dev is not None
    for k in ("x", "frac", "eps", "pRatio"):
        assert dev[k] == pytest.approx(host[k], rel=1e-12, abs=1e-15), k
    assert dev["Msep"] == pytest.approx(host["Msep"], rel=1e-12)


def synthetic_separated_state(s, last):
    """Initial state with supersonic wall flow up to column `last` and
    reversed flow from there to the exit, with a pressure dip ahead of it."""
    init = s.initialState()
    A = init["A"].reshape(s.Nr, s.Nx, 4).copy()
    B = init["B"].reshape(s.Nr, s.Nx, 4).copy()
    jw = np.asarray(s.geo["jWall"]).reshape(s.Nx, 4)[:, 0].astype(int)
    G = 2.5
    for i in range(s.iThroat + 1, s.iExit + 1):
        j = jw[i]
        rho, p = 1.0, 1.0 if i != last - 4 else 0.4
        u = 2.5 if i < last else -0.2
        A[j, i] = (rho, rho * u, 0.0, p * G + 0.5 * rho * u * u)
        B[j, i, 2] = G
    return A.reshape(-1), B.reshape(-1)


@pytest.mark.parametrize("precision", ["exact", "fast"])
def test_separation_synthetic(rn, precision):
    s = viscous(rn)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setPrecision(precision)
    g.setGeometry(s.geo)
    last = s.iExit - 8
    A, B = synthetic_separated_state(s, last)
    g.setState(A, B)
    paSi = 101325.0
    dev = g.wallSeparation(s, paSi)
    host = host_separation(rn, g, s, paSi)
    assert host is not None and dev is not None
    assert_same(dev, host)
    assert dev["x"] == pytest.approx((last + 0.5) * s.dx)
    # attached flow everywhere: no separation
    init = s.initialState()
    g.setState(init["A"], init["B"])
    assert g.wallSeparation(s, paSi) is None and host_separation(rn, g, s, paSi) is None
    g.close()


def test_separation_during_start_up(rn):
    """Sea-level start of the expansion-20 bell (over-expanded): device and
    host read-outs agree at every check."""
    s = viscous(rn)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setPrecision("exact")
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    for _ in range(6):
        g.step(250, s.P)
        assert_same(g.wallSeparation(s, 101325.0), host_separation(rn, g, s, 101325.0))
    g.close()


def oracle_derived():
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "derived.py")
    spec = importlib.util.spec_from_file_location("oracle_derived", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


RANGES = {"temp": (250.0, 3500.0), "mach": (0.0, 4.0), "schl": (0.0, 1.0), "pres": (3.0, 7.0), "dens": (-2.0, 2.0),
          "vel": (0.0, 3500.0), "vort": (0.0, 2e5), "exh": (0.0, 1.0), "flame": (250.0, 3500.0),
          "turb": (0.0, 3.0), "burn": (0.0, 1.0), "fuel": (0.0, 1.0), "ox": (0.0, 1.0), "heat": (0.0, 6.0)}


def test_derived_fields_match_shader_restatement(rn, oracle):
    """Every display field of FS_DERIVED on the device against the NumPy
    restatement of the shader, on the same state (exact precision, 60 steps of
    the viscous plume: the device state equals the oracle's, whose T2 texture
    feeds the restatement of fields 'turb' and 'heat')."""
    from rocket_nozzle_cfd_solver_b200 import solver
    from helpers import run_oracle
    D = oracle_derived()
    s = viscous(rn, 128, 48)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setPrecision("exact")
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    g.step(60, s.P)
    st = g.readAll()
    o = run_oracle(oracle, s, 60)
    ref_state = o.readAll()
    assert np.array_equal(st["A"], ref_state["A"])
    T2 = o.readT2().astype(np.float32)
    for name in solver.FIELDS:
        spec = solver.derived_spec(s, name, RANGES[name])
        dev = g.derived(spec, s.P).reshape(-1, 4)
        ref = D.derived(st["A"], st["B"], s.mask, s.Nx, s.Nr, spec, T2).reshape(-1, 4)
        np.testing.assert_allclose(dev, ref, rtol=2e-5, atol=2e-6, err_msg=name)
        assert np.all(dev[s.mask != 0] == (0, 0, 0, -1))
    assert g.derivedBuffer() != 0
    g.close()


def test_derived_turbulence_fields_need_a_step(rn):
    from rocket_nozzle_cfd_solver_b200 import solver
    s = viscous(rn, 96, 36)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    out = g.derived(solver.derived_spec(s, "turb", RANGES["turb"]), s.P).reshape(-1, 4)
    assert np.all(out[s.mask == 0, 0] == np.float32(0.0 - 0.0) / np.float32(3.0))   # T2 = 0 before any step
    with pytest.raises(rn.RnError):
        g.derived(solver.derived_spec(s, "turb", RANGES["turb"]))              # P required
    g.close()


@pytest.mark.parametrize("key", ["injShower", "injCoax", "injImpinge", "injPintle", "injHardware"])
def test_injector_table_built_on_device(rn, key):
    """The device fill of the injector table equals the host table of
    build_injector_table (bit for bit), also with a film-cooling element."""
    from rocket_nozzle_cfd_solver_b200 import configs, solver
    for film in (0, 12):
        cfg = dict(configs.preset(key, 192), film=film)
        s = rn.build_sim_setup(cfg)
        g = rn.GPUSolver(s.Nx, s.Nr)
        rn.GPUSpray(g).resize()
        g.spray.buildInjector(s.injector)
        tab = g._readRect(solver.RN_TEX_INJECTOR, 0, 0, 256, 3)
        ref = np.asarray(s.injector["tab"], np.float32)
        assert np.array_equal(tab.view(np.uint32), ref.view(np.uint32)), (key, film)
        g.close()
