"""The cut-cell geometry builder on the device (rn_build_geometry) against the
host restatement of buildCutGeometry + the geoM post-pass (cutcell.py,
simsetup.py): topology and every float plane bit-identical, over engine
presets that exercise chamber hardware (pintle, baffles, cavity), a base
body, the staircase wall model and the batched workload's grid sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cases(rn):
    from rocket_nozzle_cfd_solver_b200 import configs
    out = [("plain 256x96", configs.plain_small(256, 96)[0]),
           ("viscous 512x192", configs.viscous_plume(512, 192)[0]),
           ("spray chamber 512x192", configs.injector_spray(512, 192)[0])]
    for key in ("injPintle", "injHardware", "flight", "overexp", "coldgas", "hybrid", "upper"):
        out.append((key, configs.preset(key, 320)))
    stair = dict(configs.viscous_plume(256, 96)[0], wallModel="stair")
    out.append(("stair 256x96", stair))
    cav = dict(configs.injector_spray(384, 144)[0], cavD=20, cavW=40, baffles=3, baffleH=30, injType="pintle")
    out.append(("cavity+baffles+pintle", cav))
    rng = np.random.default_rng(5)
    for n in range(4):
        out.append((f"batched draw {n}", configs.batched_instance(rng, configs.BATCH_SIZES[n])))
    return out


@pytest.fixture(scope="module")
def setups(rn):
    return [(name, rn.build_sim_setup(cfg)) for name, cfg in cases(rn)]


def test_device_builder_bit_identical(rn, setups):
    for name, s in setups:
        g = rn.GPUSolver(s.Nx, s.Nr)
        st = g.buildGeometry(s)
        d = g.readGeometry()
        geo = s.geo
        assert np.array_equal(d["mask"], np.asarray(geo["mask"], np.uint8)), name
        for k in ("geoA", "geoG", "geoM", "jWall"):
            a = np.asarray(geo[k], np.float32)
            assert np.array_equal(d[k].view(np.uint32), a.view(np.uint32)), (name, k)
        assert st == {"nCut": geo["nCut"], "nMerged": geo["nMerged"]}, name
        g.close()


def test_device_built_geometry_steps_like_uploaded(rn, setups):
    name, s = [x for x in setups if x[0] == "viscous 512x192"][0]
    outs = []
    for dev in (False, True):
        g = rn.GPUSolver(s.Nx, s.Nr)
        g.setPrecision("exact")
        if dev:
            g.buildGeometry(s)
        else:
            g.setGeometry(s.geo)
        init = s.initialState()
        g.setState(init["A"], init["B"])
        g.step(40, s.P)
        outs.append(g.readAll())
        g.close()
    assert np.array_equal(outs[0]["A"], outs[1]["A"]) and np.array_equal(outs[0]["B"], outs[1]["B"])
