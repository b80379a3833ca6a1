"""The reference's own published simulation results, reproduced through the
CUDA path: parity pinned to numbers the reference itself produced.

The reference ships no golden vectors. Its README does publish the read-outs
its solver gave on the Medium grid (1024 x 287):

* kerolox demo, methalox shock diamonds and N2O/HTPB hybrid at sea level:
  chamber pressure, mass flow, thrust and Isp "at the exit plane after the
  start-up transient" (README.md:92-101);
* the hydrolox vacuum bell fired at sea level: wall pressure / ambient at
  separation and the separation point as a share of bell length
  (README.md:105-112);
* the injector presets at 70 bar: chamber pressure and Isp at about 2 ms of
  simulated time, the hydrolox coaxial case at 1.5 ms and the pintle at 3.5 ms
  (README.md:47-55).

Each case is set up as the app applies the preset over its default settings
(app.js:1108-1122, configs.preset) and read out with the app's protocol: the
exit column and the chamber cell read back every 20 steps (the app's steps per
frame), converted by exitPerformance/cellPrimSI (simsetup.js:314-348) and
time-averaged with the app's 60 us exponential average (processMeasurements,
app.js:519-532); separation through wallSeparation with the app's 0.2 position
smoothing (app.js:567-571). Plume cases are read at 1.5 ms, the separation at
3 ms ("about 3 ms to settle", README.md:155), injector cases at the README's
times.

Tolerances. The README does not state when in the run it read its values, and
between 1 and 2 ms the read-outs still drift as the chamber relaxes onto its
target (this path: hybrid chamber pressure 30.4 -> 29.7 bar, demo thrust
13.30 -> 13.13 kN); the reference's own figures sit inside that drift. The
chaotic plume and chamber also decorrelate from a run whose last-bit rounding
differs (WebGL2 highp shaders against sm_100a FP32), which the 60 us average
only partly smooths. Bars: 3 % on chamber pressure, mass flow and Isp, 5 % on
thrust (the quantity that drifts most); separation p/pa within 0.05 and its
position within 5 % of bell length; injector chamber pressure and Isp within
5 %. Isp is F / (mdot g0) of the averaged thrust and mass flow (the app's
averaged Isp equals it once settled)."""
import math

import pytest

pytestmark = pytest.mark.gpu

AVG_TAU = 6e-5       # app.js:517
FRAME = 20           # steps per frame (app settings, app.js:23)
G0 = 9.80665

PLUME = {            # README.md:92-101 (simulated rows)
    "demo": dict(pc_bar=195.1, mdot=4.46, F_kN=13.22, Isp=301.0),
    "diamonds": dict(pc_bar=90.2, mdot=3.44, F_kN=9.83, Isp=289.0),
    "hybrid": dict(pc_bar=30.6, mdot=1.42, F_kN=3.10, Isp=220.0),
}
INJECTOR = {         # README.md:47-55: (preset, propellant override, time in ms, chamber bar, Isp s)
    "shower_kerolox": ("injShower", None, 2.0, 64.6, 272.0),
    "impinge_kerolox": ("injImpinge", None, 2.0, 65.8, 281.0),
    "coax_methalox": ("injCoax", None, 2.0, 68.3, 287.0),
    "coax_hydrolox": ("injCoax", "hydrolox", 1.5, 68.2, 348.0),
    "hardware_kerolox": ("injHardware", None, 2.0, 65.5, 283.0),
    "pintle_kerolox": ("injPintle", None, 3.5, 63.5, 264.0),
}


def preset_cfg(key, prop=None):
    from rocket_nozzle_cfd_solver_b200 import configs
    from rocket_nozzle_cfd_solver_b200.physics import PROPELLANTS
    cfg = configs.preset(key, 1024)
    if prop:                                     # the app's propellant switch (app.js:1086-1094)
        p = PROPELLANTS[prop]
        cfg.update(prop=prop, Tc=p["Tc"], gamma=p["gamma"], Mw=p["Mw"], qAb=p["qAb"], sAir=p["sAir"])
        if p.get("spray"):
            cfg["OF"] = p["spray"]["OF"]
    return cfg


def app_readouts(rn, cfg, t_ms, separation=False):
    """Run the preset to t_ms of simulated time with the app's read-out
    protocol; returns the averaged exit/chamber read-outs (and separation)."""
    from rocket_nozzle_cfd_solver_b200 import simsetup, solver
    from rocket_nozzle_cfd_solver_b200.physics import atmosphere
    s = rn.build_sim_setup(cfg)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    if s.injector is not None:
        rn.GPUSpray(g).resize()
        g.spray.setInjector(s.injector)
    pa = atmosphere(cfg["alt"])["p"]
    perf = chamber = sep = None
    hold, sim_t = 0, 0.0
    while sim_t * 1e3 < t_ms:
        g.step(FRAME, s.P)
        t_prev, sim_t = sim_t, float(g.readStepInfo()[2]) * s.tScale
        p_now = simsetup.exit_performance(s, g.readColumn(s.iExit))
        ch = g.readCell(s.iChamber, 0)
        c_now = simsetup.cell_prim_si(s, ch["A"], ch["B"])
        if perf is None:
            perf, chamber = dict(p_now), dict(c_now)
        else:
            a = 1 - math.exp(-max(0.0, sim_t - t_prev) / AVG_TAU)
            for k in perf:
                perf[k] += (p_now[k] - perf[k]) * a
            for k in chamber:
                chamber[k] += (c_now[k] - chamber[k]) * a
        if separation:
            g.drawWallRow()
            row = g._readRect(solver.RN_TEX_WALLROW, 0, 0, s.Nx, 1)
            now = simsetup.wall_separation(s, row, pa)
            if now:
                sep = dict(now) if sep is None else dict(now, x=sep["x"] + (now["x"] - sep["x"]) * 0.2,
                                                        frac=sep["frac"] + (now["frac"] - sep["frac"]) * 0.2)
                hold = 12
            else:
                hold -= 1
                if hold <= 0:
                    sep = None
    g.close()
    out = dict(t_ms=sim_t * 1e3, pc_bar=chamber["p"] / 1e5, mdot=perf["mdot"], F_kN=perf["F"] / 1e3,
               Isp=perf["F"] / (perf["mdot"] * G0))
    if separation:
        out["sep"] = sep
    return out


def rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.parametrize("key", sorted(PLUME))
def test_plume_presets_match_readme(rn, key):
    got = app_readouts(rn, preset_cfg(key), 1.5)
    ref = PLUME[key]
    print(key, {k: round(v, 4) for k, v in got.items()}, "README", ref)
    assert rel(got["pc_bar"], ref["pc_bar"]) <= 0.03, got
    assert rel(got["mdot"], ref["mdot"]) <= 0.03, got
    assert rel(got["Isp"], ref["Isp"]) <= 0.03, got
    assert rel(got["F_kN"], ref["F_kN"]) <= 0.05, got


def test_overexpanded_bell_separation_matches_readme(rn):
    """Hydrolox vacuum bell (120 bar, eps 64) at sea level: p/pa 0.49 at 58 %
    of the bell (README.md:105-112)."""
    got = app_readouts(rn, preset_cfg("overexp"), 3.0, separation=True)
    print("overexp", got)
    assert got["sep"] is not None, "no separation found"
    assert abs(got["sep"]["pRatio"] - 0.49) <= 0.05, got
    assert abs(got["sep"]["frac"] - 0.58) <= 0.05, got


@pytest.mark.parametrize("case", sorted(INJECTOR))
def test_injector_presets_match_readme(rn, case):
    key, prop, t_ms, pc, isp = INJECTOR[case]
    got = app_readouts(rn, preset_cfg(key, prop), t_ms)
    print(case, {k: round(v, 4) for k, v in got.items()}, "README", pc, isp)
    assert rel(got["pc_bar"], pc) <= 0.05, got
    assert rel(got["Isp"], isp) <= 0.05, got
