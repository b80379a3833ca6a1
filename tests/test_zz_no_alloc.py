"""rn_integrals_static: the FP64 read-outs for callers that cannot allocate
device memory when they need them (an application that reserves the whole
device memory budget up front, or a latency-critical loop that cannot take
cudaMalloc's implicit synchronisation). It reads buffers the caller owns and
keeps its scratch in a static device array, so it is checked here against
rn_integrals (which stages its sums in memory the solver handle allocated) on
two calls in a row, through the C-ABI. Collected last on purpose: it must pass
alone in a fresh process and after every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12          # both are compensated FP64 sums; only the summation order differs


def spec_for(rn, s):
    from rocket_nozzle_cfd_solver_b200 import solver
    sp = solver.RnIntegralSpec()
    sp.iExit, sp.jExit, sp.iThroat, sp.iChamber = s.iExit, s.jExit, s.iThroat, s.iChamber
    sp.dx = s.dx
    sp.pAmb = s.P["amb"][3]
    for k in range(3):
        sp.Rs[k] = s.P["Rs"][k]
    sp.RaN = s.P["RaN"]
    sp.inj = 1 if s.P["inj"] else 0
    return sp


def static_call(rn, s, state, stepinfo, Nr=None, stream=None):
    """rn_integrals_static on device copies of the state the caller owns;
    ``stream`` is a torch.cuda.Stream or None (the legacy default stream)."""
    import torch
    from rocket_nozzle_cfd_solver_b200 import solver
    dev = torch.device("cuda:0")
    A = torch.from_numpy(np.ascontiguousarray(state["A"], dtype=np.float32)).to(dev)
    B = torch.from_numpy(np.ascontiguousarray(state["B"], dtype=np.float32)).to(dev)
    geoA = torch.from_numpy(np.ascontiguousarray(s.geo["geoA"], dtype=np.float32)).to(dev)
    mask = torch.from_numpy(np.ascontiguousarray(s.mask, dtype=np.uint8)).to(dev)
    st = torch.from_numpy(np.ascontiguousarray(stepinfo, dtype=np.float32)).to(dev)
    torch.cuda.synchronize()
    out = solver.RnIntegralsOut()
    rc = solver.lib().rn_integrals_static(A.data_ptr(), B.data_ptr(), geoA.data_ptr(), mask.data_ptr(), s.Nx,
                                          s.Nr if Nr is None else Nr, st.data_ptr(), ctypes.byref(spec_for(rn, s)),
                                          ctypes.byref(out), None if stream is None else stream.cuda_stream)
    return rc, {n: getattr(out, n) for n, _ in solver.RnIntegralsOut._fields_}


def test_static_integrals_match_rn_integrals_on_two_calls(rn):
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.viscous_plume(128, 48)[0])
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    g.step(600, s.P)
    for call in range(2):
        ref = g.integrals(s)                      # the existing entry point
        rc, got = static_call(rn, s, g.readAll(), g.readStepInfo())
        assert rc == 0, rn.solver.lib().rn_last_error()
        for k, v in ref.items():
            assert got[k] == pytest.approx(v, rel=REL, abs=1e-300), (call, k)
        assert ref["throat_mdot"] > 0.0 and ref["A"] > 0.0 and ref["chamber_p"] > 0.0
        g.step(300, s.P)                          # second call sees a different state
    g.close()


def test_static_integrals_reject_oversize(rn):
    from rocket_nozzle_cfd_solver_b200 import configs, solver
    s = rn.build_sim_setup(configs.plain_small(96, 36)[0])
    init = s.initialState()
    rc, _ = static_call(rn, s, init, np.zeros(4, np.float32), Nr=4097)
    assert rc == -1
    assert b"static scratch" in solver.lib().rn_last_error()


def test_static_integrals_on_a_caller_stream(rn):
    """The caller's own (non-default) stream: same read-outs as rn_integrals."""
    import torch
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.viscous_plume(128, 48)[0])
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    g.step(400, s.P)
    ref = g.integrals(s)
    st = torch.cuda.Stream()
    rc, got = static_call(rn, s, g.readAll(), g.readStepInfo(), stream=st)
    assert rc == 0, rn.solver.lib().rn_last_error()
    for k, v in ref.items():
        assert got[k] == pytest.approx(v, rel=REL, abs=1e-300), k
    g.close()


def test_static_integrals_refuse_a_capturing_stream(rn):
    """A stream under capture is refused before anything is queued on it."""
    import torch
    from rocket_nozzle_cfd_solver_b200 import configs, solver
    s = rn.build_sim_setup(configs.plain_small(96, 36)[0])
    init = s.initialState()
    dev = torch.device("cuda:0")
    bufs = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in
            (np.asarray(init["A"], np.float32), np.asarray(init["B"], np.float32),
             np.asarray(s.geo["geoA"], np.float32), np.asarray(s.mask, np.uint8), np.zeros(4, np.float32))]
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    out = solver.RnIntegralsOut()
    L = solver.lib()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=st, capture_error_mode="thread_local"):
        bufs[4].add_(0.0)                        # the capture holds one op of the caller's
        rc = L.rn_integrals_static(bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(), bufs[3].data_ptr(),
                                   s.Nx, s.Nr, bufs[4].data_ptr(), ctypes.byref(spec_for(rn, s)), ctypes.byref(out),
                                   st.cuda_stream)
    assert rc == -1
    assert b"captured" in L.rn_last_error()
    graph.replay()                               # the caller's capture stayed valid
    torch.cuda.synchronize()
    del graph
