"""The FP64 residual and the solve server (continuous batching), through
librn.so.

The residual is checked against a NumPy FP64 evaluation of the same formula
on read-back states. The server's results must not depend on the mix: in
exact precision every solve's final state and FP64 read-outs are
bit-identical to the same solve stepped alone on its own handle, whatever
else was admitted beside it and whenever it was admitted."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup_of(rn, kind, Nx, Nr):
    from rocket_nozzle_cfd_solver_b200 import configs
    f = {"plain": configs.plain_small, "viscous": configs.viscous_plume, "spray": configs.injector_spray}[kind]
    return rn.build_sim_setup(f(Nx, Nr)[0])


def alone(rn, s, steps, precision="exact"):
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setPrecision(precision)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    if s.injector is not None:
        rn.GPUSpray(g).resize()
        g.spray.setInjector(s.injector)
    g.step(steps, s.P)
    out = g.readAll()
    integ = g.integrals(s)
    g.close()
    return out, integ


def numpy_residual(A0, A1, mask, span):
    fluid = mask.reshape(-1) == 0
    d = (A1.reshape(-1, 4).astype(np.float64) - A0.reshape(-1, 4).astype(np.float64))[fluid]
    return np.sqrt((d * d).sum(axis=0) / fluid.sum()) / span, int(fluid.sum())


def test_residual_matches_numpy(rn):
    s = setup_of(rn, "viscous", 128, 48)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    g.step(30, s.P)
    A0, t0 = g.readAll()["A"], g.readStepInfo()[2]
    g.residualMark()
    g.step(1, s.P)
    A1, t1 = g.readAll()["A"], g.readStepInfo()[2]
    r = g.residual()
    ref, nf = numpy_residual(A0, A1, s.mask, float(t1) - float(t0))
    assert r["cells"] == nf and r["span"] == pytest.approx(float(t1) - float(t0), rel=1e-12)
    got = np.array([r["rho"], r["rhou"], r["rhov"], r["E"]])
    assert np.all(got > 0)
    np.testing.assert_allclose(got, ref, rtol=1e-12)
    assert g.residual() == r                                 # deterministic
    g.close()


def test_residual_needs_a_mark(rn):
    s = setup_of(rn, "plain", 96, 36)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    with pytest.raises(rn.RnError):
        g.residual()
    g.close()


def test_server_results_same_alone_and_in_mix(rn):
    """Solves of three physics classes and uneven sizes, admitted under a
    budget that holds only some at a time, arriving in two waves: each ends
    bit-identical to the same solve stepped alone."""
    cases = [("plain", 96, 36), ("plain", 160, 60), ("viscous", 128, 48), ("plain", 256, 96),
             ("viscous", 96, 36), ("spray", 96, 36)]
    ss = [setup_of(rn, *c) for c in cases]
    steps = 120
    budget = sum(sorted(rn.SolveServer.solve_bytes(s.Nx, s.Nr) for s in ss)[-3:])
    srv = rn.SolveServer(budget_bytes=budget, check_every=30, precision="exact")
    ids = [srv.submit(s, drop=0, t_end_s=0, max_steps=steps) for s in ss[:3]]
    time.sleep(0.05)
    ids += [srv.submit(s, drop=0, t_end_s=0, max_steps=steps) for s in ss[3:]]
    res = [srv.wait(i, timeout_s=300, state=True) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["admitted"] == len(ss) and st["failed"] == 0 and st["bytes_used"] == 0
    for s, r in zip(ss, res):
        assert r is not None and r["status"] == "max_steps" and r["steps"] == steps
        out, integ = alone(rn, s, steps)
        assert np.array_equal(r["A"], out["A"]) and np.array_equal(r["B"], out["B"])
        assert r["integrals"] == integ
        assert r["submit_ms"] <= r["admit_ms"] <= r["done_ms"]
        assert r["residual0"] > 0 and r["residual"] > 0


def test_server_budget_and_rejection(rn):
    ss = [setup_of(rn, "plain", 96, 36), setup_of(rn, "plain", 128, 48), setup_of(rn, "plain", 96, 36)]
    big = setup_of(rn, "plain", 512, 192)
    one = max(rn.SolveServer.solve_bytes(s.Nx, s.Nr) for s in ss)
    srv = rn.SolveServer(budget_bytes=one, check_every=20)
    ids = [srv.submit(s, drop=0, t_end_s=0, max_steps=200) for s in ss]
    rid_big = srv.submit(big, drop=0, t_end_s=0, max_steps=20)
    peak = 0
    t0 = time.time()
    while srv.stats()["admitted"] < len(ss) and time.time() - t0 < 120:
        peak = max(peak, srv.stats()["active"])
        time.sleep(0.001)
    res = [srv.wait(i, timeout_s=120) for i in ids]
    rb = srv.wait(rid_big, timeout_s=120)
    srv.close()
    assert peak <= 1
    assert all(r["status"] == "max_steps" and r["steps"] == 200 for r in res)
    assert rb["status"] == "rejected"
    # one at a time, in arrival order
    assert res[0]["done_ms"] <= res[1]["admit_ms"] and res[1]["done_ms"] <= res[2]["admit_ms"]


def test_server_time_and_poll(rn):
    s = setup_of(rn, "viscous", 128, 48)
    srv = rn.SolveServer(check_every=25)
    rid = srv.submit(s, drop=0, t_end_s=2e-5, max_steps=5000)   # 20 us: a few dozen steps
    r = None
    t0 = time.time()
    while r is None and time.time() - t0 < 120:
        r = srv.poll(rid)
        time.sleep(0.001)
    srv.close()
    assert r is not None
    assert r["status"] == "time" and r["t"] * s.tScale >= 2e-5 and r["steps"] % 25 == 0
    assert np.isfinite(r["integrals"]["F"]) and r["integrals"]["t"] == pytest.approx(r["t"], rel=1e-6)


def test_server_cell_cap(rn):
    """max_active_cells admits solves while their grids fit the cap (always at
    least one); results are unchanged by the admission order."""
    ss = [setup_of(rn, "plain", 128, 48), setup_of(rn, "plain", 128, 48), setup_of(rn, "plain", 96, 36)]
    srv = rn.SolveServer(check_every=20, max_active_cells=128 * 48 + 96 * 36, precision="exact")
    ids = [srv.submit(s, drop=0, t_end_s=0, max_steps=100) for s in ss]
    peak = 0
    t0 = time.time()
    while srv.stats()["admitted"] < len(ss) and time.time() - t0 < 120:
        peak = max(peak, srv.stats()["active"])
        time.sleep(0.0005)
    res = [srv.wait(i, timeout_s=120, state=True) for i in ids]
    srv.close()
    assert peak <= 2
    assert res[0]["done_ms"] <= res[1]["admit_ms"]          # the second 128x48 waits for the first
    for s, r in zip(ss, res):
        out, _ = alone(rn, s, 100)
        assert np.array_equal(r["A"], out["A"])


def test_server_isolates_failing_requests(rn):
    """A request whose setup fails (a geometry the library rejects), one whose
    admission allocation fails and one whose first tick fails (host-side
    injections of an allocation failure) are each evicted alone with status
    'failed'; the other solves finish bit-identical to the same solves
    stepped alone, and the server keeps accepting work."""
    import copy
    good = [setup_of(rn, "plain", 96, 36), setup_of(rn, "viscous", 128, 48), setup_of(rn, "plain", 128, 48)]
    bad_geo = copy.copy(setup_of(rn, "plain", 96, 36))
    geo = dict(bad_geo.geo)
    geoM = np.array(geo["geoM"], dtype=np.float32).reshape(-1, 4)
    k = int(np.flatnonzero(np.asarray(geo["mask"]) == 0)[40])
    geoM[k, 0] = 2.0                                  # a host two cells away: rn_set_geometry rejects it
    geo["geoM"] = geoM.ravel()
    bad_geo["geo"] = geo
    steps = 80
    srv = rn.SolveServer(check_every=20, precision="exact")
    ids = {"g0": srv.submit(good[0], drop=0, t_end_s=0, max_steps=steps)}
    ids["setup"] = srv.submit(bad_geo, drop=0, t_end_s=0, max_steps=steps)
    srv.inject("admit")
    ids["admit"] = srv.submit(good[1], drop=0, t_end_s=0, max_steps=steps)
    ids["g1"] = srv.submit(good[1], drop=0, t_end_s=0, max_steps=steps)
    srv.inject("tick")
    ids["tick"] = srv.submit(good[2], drop=0, t_end_s=0, max_steps=steps)
    ids["g2"] = srv.submit(good[2], drop=0, t_end_s=0, max_steps=steps)
    res = {k: srv.wait(v, timeout_s=300, state=True) for k, v in ids.items()}
    later = srv.submit(good[0], drop=0, t_end_s=0, max_steps=steps)   # still serving
    r_later = srv.wait(later, timeout_s=300, state=True)
    st = srv.stats()
    srv.close()
    for k in ("setup", "admit", "tick"):
        assert res[k]["status"] == "failed", (k, res[k]["status"])
    assert st["failed"] == 0 and st["evicted"] == 3 and st["bytes_used"] == 0
    for k, s in (("g0", good[0]), ("g1", good[1]), ("g2", good[2]), ("later", good[0])):
        r = r_later if k == "later" else res[k]
        assert r["status"] == "max_steps" and r["steps"] == steps, k
        out, integ = alone(rn, s, steps)
        assert np.array_equal(r["A"], out["A"]) and np.array_equal(r["B"], out["B"]), k
        assert r["integrals"] == integ, k
